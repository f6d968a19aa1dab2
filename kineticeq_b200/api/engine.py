"""Engine mirror (api/engine.py:24-116): fills default model/scheme params,
builds the state and the stepper through the registry, and runs
``n_steps`` calls of the stepper with the reference's progress/benchlog
printing every n_steps//10 steps."""
from __future__ import annotations

import logging
from dataclasses import replace

from ..params.registry import default_model_cfg, default_scheme_params, expected_model_cfg_type
from ..schemes.registry import build_stepper
from ..state import build_state
from .config import Config, LogLevel

logger = logging.getLogger("kineticEQ")


class Result:
    """Empty result object, as api/result.py:5-8."""


def _format_kv(d) -> str:
    if d is None:
        return ""
    items = d.items() if hasattr(d, "items") else vars(d).items()
    return "\n".join(f"  {k}: {v}" for k, v in items)


def apply_logging(cfg: Config) -> None:
    level = {LogLevel.DEBUG: logging.DEBUG, LogLevel.INFO: logging.INFO,
             LogLevel.WARNING: logging.WARNING, LogLevel.ERROR: logging.ERROR}[cfg.log_level]
    logger.setLevel(level)
    if not logger.handlers:
        h = logging.StreamHandler()
        h.setFormatter(logging.Formatter("%(levelname)s %(name)s: %(message)s"))
        logger.addHandler(h)


class Engine:
    def __init__(self, config: Config, apply_logging_flag: bool = True):
        self.config = config
        if self.config.model_cfg is None:
            self.config = replace(self.config, model_cfg=default_model_cfg(self.config.model))
        else:
            t = expected_model_cfg_type(self.config.model)
            if not isinstance(self.config.model_cfg, t):
                raise TypeError(f"model_cfg type mismatch: expected {t.__name__}, "
                                f"got {type(self.config.model_cfg).__name__}")
        if self.config.model_cfg.scheme_params is None:
            sp = default_scheme_params(self.config.model, self.config.scheme)
            if sp is not None:
                self.config = replace(self.config,
                                      model_cfg=replace(self.config.model_cfg, scheme_params=sp))
        if apply_logging_flag:
            apply_logging(self.config)
        logger.info("Engine: model=%s scheme=%s backend=%s device=%s",
                    self.config.model_name, self.config.scheme_name,
                    self.config.backend_name, self.config.device)
        if str(self.config.device).startswith("cuda"):
            import torch

            if not torch.cuda.is_available():
                raise RuntimeError("device='cuda' requested but CUDA is not available")
        self.state = build_state(self.config)
        self.stepper = build_stepper(self.config, self.state)

    def run(self) -> Result:
        n_steps = self.config.model_cfg.time.n_steps
        dt = self.config.model_cfg.time.dt
        interval = max(1, n_steps // 10)
        for step in range(n_steps):
            self.stepper(step)
            if step % interval == 0:
                bl = getattr(self.stepper, "benchlog", None)
                if bl and logger.isEnabledFor(logging.INFO):
                    logger.info("%s\nt=%.3f", _format_kv(bl), step * dt)
        return Result()


def run(config: Config) -> Result:
    return Engine(config, apply_logging_flag=True).run()
