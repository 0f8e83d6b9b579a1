"""The reference's Python module ``openTM`` (main.cpp:93-118, a pybind11 binding of runInstance
and wrapper_homo, main.cpp:17-62), over this library's design driver.

    import opentm_b200.openTM as openTM
    rho = openTM.runInstance(64, [1, 1e-4], [0.3, 0.2, 0.1, 0.1, 0.05, 0.05], openTM.InitWay.IWP,
                             openTM.Model.oc)

Where the reference prints a message and exits (wrong list lengths), these raise ValueError.
runInstance accepts further DesignConfig fields as keywords (max_iter, seed, ...), which the
reference only sets through HomoConfig::init().
"""
from __future__ import annotations

from .driver import DesignConfig, InitWay, Model, Symmetry, run_custom

__all__ = ["InitWay", "Model", "Symmetry", "runInstance", "homo"]


def _config(reso, heat_ratios, target_ratio, model) -> DesignConfig:
    heat_ratios = list(heat_ratios)
    target_ratio = list(target_ratio)
    if len(heat_ratios) != 2:
        raise ValueError("Input wrong size of heat_ratios")
    if len(target_ratio) < 6:
        raise ValueError("target_ratio needs 6 values")
    return DesignConfig(reso=int(reso), heatRatio=tuple(float(v) for v in heat_ratios),
                        target_tensor=tuple(float(v) for v in target_ratio[:6]), model=Model(model))


def runInstance(reso: int, heat_ratios, target_ratio, initway: InitWay = InitWay.IWP, model: Model = Model.mma,
                **overrides) -> list[float]:
    """runInstance (main.cpp:45-62): initialise, run the design loop, return the density."""
    cfg = _config(reso, heat_ratios, target_ratio, model)
    cfg.winit = InitWay(initway)
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise TypeError(f"unknown configuration field {k}")
        setattr(cfg, k, v)
    rho, _ = run_custom(cfg)
    return rho.ravel().tolist()


class homo:
    """wrapper_homo (main.cpp:17-44): setDensity, setConfig, optimize."""

    def __init__(self):
        self.config = DesignConfig()
        self.rho = None
        self.info = None

    def setDensity(self, rho) -> None:
        self.rho = [float(v) for v in rho]

    def setConfig(self, reso: int, heat_ratios, target_ratio, model: Model = Model.oc) -> None:
        self.config = _config(reso, heat_ratios, target_ratio, model)

    def optimize(self) -> list[float]:
        n = self.config.reso
        if self.rho is None or len(self.rho) != n ** 3:
            raise ValueError(f"setDensity needs {n ** 3} values for resolution {n}")
        rho, self.info = run_custom(self.config, rho0=self.rho)
        return rho.ravel().tolist()
