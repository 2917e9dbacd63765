"""Builds ``mpc_request_t`` values from montepath-style config mappings.

Key names and aliases follow the reference's PyO3 bridge
(crates/montepath-python/src/lib.rs:311-511, ``fill_gbm_fields`` /
``fill_path_fields`` at lib.rs:652-678): ``s0``/``spot``, ``k``/``strike``,
``r``/``rate``, ``sigma``/``volatility``, ``t``/``maturity``,
``n_paths``/``paths``, ``n_steps``/``steps``, and the Heston, Merton,
basket, LSM and MLMC fields of their configs.  Unspecified fields take the
Rust ``Default`` values (``mpc_request_defaults``).
"""

from __future__ import annotations

import ctypes
from typing import Any, Callable, Mapping

from . import abi


class ConfigError(ValueError):
    """A config value that cannot be mapped onto a request."""


def _lookup(cfg: Mapping[str, Any], keys: tuple[str, ...]):
    for key in keys:
        if key in cfg and cfg[key] is not None:
            return cfg[key]
    return None


def _enum(value: Any, table: Mapping[str, int], name: str) -> int:
    if isinstance(value, int):
        return value
    key = str(value).lower()
    if key not in table:
        raise ConfigError(f"{name} '{value}' is not one of {sorted(table)}")
    return table[key]


def defaults(workload: int) -> abi.Request:
    req = abi.Request()
    status = abi.load_library().mpc_request_defaults(ctypes.byref(req), workload)
    if status != abi.OK:
        raise ConfigError(f"unknown workload {workload}")
    return req


def make_request(workload: str | int, config: Mapping[str, Any] | None = None, *,
                 defaults: Callable[[int], abi.Request] | None = None, **overrides: Any) -> abi.Request:
    """Request for `workload` (a name of ``abi.WORKLOADS`` or its code) from a config mapping.

    `defaults(code)` supplies the starting request (the library's
    ``mpc_request_defaults`` unless given)."""

    cfg: dict[str, Any] = dict(config or {})
    cfg.update(overrides)
    code = abi.WORKLOADS[workload] if isinstance(workload, str) else int(workload)
    req = (defaults or globals()["defaults"])(code)

    def f64(attr: str, *keys: str) -> None:
        value = _lookup(cfg, keys or (attr,))
        if value is not None:
            setattr(req, attr, float(value))

    def u64(attr: str, *keys: str) -> None:
        value = _lookup(cfg, keys or (attr,))
        if value is not None:
            value = int(value)
            if value < 0:
                raise ConfigError(f"{attr} must be >= 0")
            setattr(req, attr, value)

    f64("s0", "s0", "spot")
    f64("k", "k", "strike")
    f64("r", "r", "rate")
    f64("sigma", "sigma", "volatility")
    f64("t", "t", "maturity")
    f64("barrier")
    u64("n_paths", "n_paths", "paths")
    u64("n_steps", "n_steps", "steps")
    u64("seed")
    u64("n_threads")
    for attr, table, keys in (
        ("technique", abi.TECHNIQUES, ("technique",)),
        ("sampling", abi.SAMPLINGS, ("sampling",)),
        ("method", abi.METHODS, ("method",)),
        ("precision", abi.PRECISIONS, ("precision",)),
    ):
        value = _lookup(cfg, keys)
        if value is not None:
            setattr(req, attr, _enum(value, table, attr))
    model = _lookup(cfg, ("model",))
    if model is not None:
        req.model = _enum(model, {"gbm": abi.MODEL_GBM, "heston": abi.MODEL_HESTON, "merton": abi.MODEL_MERTON}, "model")
    # Heston (lib.rs:443-460)
    f64("v0", "v0", "initial_variance")
    f64("kappa", "kappa", "mean_reversion")
    f64("theta", "theta", "long_run_variance")
    f64("vol_of_vol", "vol_of_vol", "xi")
    # Merton (lib.rs:462-479)
    f64("jump_intensity")
    f64("jump_mean")
    f64("jump_volatility")
    if code == abi.WORKLOAD_BASKET_CALL:
        _fill_basket(req, cfg)
    else:
        f64("rho", "rho", "correlation")
    # LSM
    u64("basis_degree")
    steps = _lookup(cfg, ("exercise_steps",))
    if steps is not None:
        steps = [int(s) for s in steps]
        if len(steps) > abi.MAX_EXERCISE_DATES:
            raise ConfigError("at most 64 exercise dates")
        req.n_exercise = len(steps)
        for i, s in enumerate(steps):
            req.exercise_steps[i] = s
    # MLMC (lib.rs:490-507 plus the tolerance config of cpu.rs:1611-1630)
    u64("base_steps")
    u64("levels")
    u64("refinement_factor")
    u64("scramble_replicates")
    u64("pilot_paths_per_level")
    u64("min_step_updates")
    u64("max_step_updates")
    f64("target_stderr")
    ppl = _lookup(cfg, ("paths_per_level",))
    if ppl is not None:
        ppl = [int(p) for p in ppl]
        if len(ppl) > abi.MAX_LEVELS:
            raise ConfigError("at most 16 MLMC levels")
        for i in range(abi.MAX_LEVELS):
            req.paths_per_level[i] = ppl[i] if i < len(ppl) else 0
    u64("block_size")
    u64("paths_per_thread")
    return req


def _fill_basket(req: abi.Request, cfg: Mapping[str, Any]) -> None:
    """Two-asset reference keys (lib.rs:375-399) or d-asset lists."""

    spots = _lookup(cfg, ("spots",))
    if spots is not None:
        d = len(spots)
        if not 1 <= d <= abi.MAX_ASSETS:
            raise ConfigError("a basket has 1..=8 assets")
        sigmas = _lookup(cfg, ("sigmas", "volatilities")) or [req.sigma] * d
        weights = _lookup(cfg, ("weights",)) or [1.0 / d] * d
        corr = _lookup(cfg, ("corr", "correlation", "rho"))
        if corr is None:
            corr = 0.0
        req.n_assets = d
        for i in range(d):
            req.spots[i] = float(spots[i])
            req.sigmas[i] = float(sigmas[i])
            req.weights[i] = float(weights[i])
        for i in range(d):
            for j in range(d):
                if isinstance(corr, (int, float)):
                    value = 1.0 if i == j else float(corr)
                else:
                    value = float(corr[i][j])
                req.corr[i * d + j] = value
        return
    values = {
        "s01": _lookup(cfg, ("s01", "spot_1", "spot1")),
        "s02": _lookup(cfg, ("s02", "spot_2", "spot2")),
        "sigma1": _lookup(cfg, ("sigma1", "volatility_1", "volatility1")),
        "sigma2": _lookup(cfg, ("sigma2", "volatility_2", "volatility2")),
        "w1": _lookup(cfg, ("weight1", "weight_1")),
        "w2": _lookup(cfg, ("weight2", "weight_2")),
        "rho": _lookup(cfg, ("rho", "correlation")),
    }
    req.n_assets = 2
    if values["s01"] is not None:
        req.spots[0] = float(values["s01"])
    if values["s02"] is not None:
        req.spots[1] = float(values["s02"])
    if values["sigma1"] is not None:
        req.sigmas[0] = float(values["sigma1"])
    if values["sigma2"] is not None:
        req.sigmas[1] = float(values["sigma2"])
    if values["w1"] is not None:
        req.weights[0] = float(values["w1"])
    if values["w2"] is not None:
        req.weights[1] = float(values["w2"])
    if values["rho"] is not None:
        rho = float(values["rho"])
        req.corr[1] = rho
        req.corr[2] = rho
    req.corr[0] = 1.0
    req.corr[3] = 1.0


def request_to_dict(req: abi.Request) -> dict[str, Any]:
    out: dict[str, Any] = {}
    for name, ctype in req._fields_:
        if name.startswith("_"):
            continue
        value = getattr(req, name)
        if hasattr(value, "__len__") and not isinstance(value, (bytes, str)):
            value = list(value)
        out[name] = value
    return out


def copy_request(req: abi.Request) -> abi.Request:
    out = abi.Request()
    ctypes.memmove(ctypes.byref(out), ctypes.byref(req), ctypes.sizeof(abi.Request))
    return out


def heston_request(**kw: Any) -> abi.Request:
    kw.setdefault("model", "heston")
    return make_request("european_call", kw)


def merton_request(**kw: Any) -> abi.Request:
    kw.setdefault("model", "merton")
    return make_request("european_call", kw)


def correlation_matrix(d: int, rho: float) -> list[list[float]]:
    return [[1.0 if i == j else rho for j in range(d)] for i in range(d)]

