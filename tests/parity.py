"""Photon-by-photon comparison of GPU records with oracle records."""
from __future__ import annotations

import numpy as np

# acceptance bounds of the path: positions within 1e-4 mm, directions within 1e-5 rad
POS_TOL_M = 1e-7
DIR_TOL_RAD = 1e-5
PATH_TOL_M = 1e-7
VALUE_RTOL = 1e-4


def _angle(a, b):
    na = np.linalg.norm(a, axis=-1)
    nb = np.linalg.norm(b, axis=-1)
    c = np.sum(a * b, axis=-1) / np.maximum(na * nb, 1e-30)
    return np.arccos(np.clip(c, -1.0, 1.0))


def compare_records(gpu, ref) -> dict:
    """Return per-photon match flags and diagnostics."""
    n = len(ref)
    same_events = (gpu["end"] == ref["end"]) & (gpu["draws"] == ref["draws"]) & (gpu["depth"] == ref["depth"]) & (
        gpu["n_splats"] == ref["n_splats"])
    pos_err = np.max(np.abs(gpu["pos"].astype(np.float64) - ref["pos"].astype(np.float64)), axis=1)
    dir_err = _angle(gpu["dir"].astype(np.float64), ref["dir"].astype(np.float64))
    path_err = np.abs(gpu["total_optical"] - ref["total_optical"])
    k = np.minimum(ref["n_splats"], gpu["splats"].shape[1])
    spl_pos = np.zeros(n)
    spl_path = np.zeros(n)
    spl_val = np.zeros(n)
    spl_depth = np.ones(n, dtype=bool)
    for i in range(gpu["splats"].shape[1]):
        m = (i < k) & same_events
        if not m.any():
            continue
        gs, rs = gpu["splats"][:, i], ref["splats"][:, i]
        e = np.max(np.abs(gs["p"].astype(np.float64) - rs["p"].astype(np.float64)), axis=1)
        spl_pos = np.where(m, np.maximum(spl_pos, e), spl_pos)
        spl_path = np.where(m, np.maximum(spl_path, np.abs(gs["pathlength"] - rs["pathlength"])), spl_path)
        rel = np.abs(gs["value"] - rs["value"]) / np.maximum(np.abs(rs["value"]), 1e-30)
        spl_val = np.where(m, np.maximum(spl_val, rel), spl_val)
        spl_depth &= ~m | (gs["depth"] == rs["depth"])
    # the acceptance bounds of the path: every event equal, positions (end and splats) within 1e-4 mm,
    # directions within 1e-5 rad, path lengths within 1e-4 mm
    ok_geom = same_events & (pos_err <= POS_TOL_M) & (dir_err <= DIR_TOL_RAD) & (path_err <= PATH_TOL_M) & (
        spl_pos <= POS_TOL_M) & (spl_path <= PATH_TOL_M) & spl_depth
    # and, stricter, every splat value within 1e-4 relative (its exp(-sigma_t d) factor compounds the
    # FP32 rounding of metres of internally reflected path)
    ok = ok_geom & (spl_val <= VALUE_RTOL)
    return {"ok": ok, "ok_geom": ok_geom, "same_events": same_events, "pos_err": pos_err, "dir_err": dir_err,
            "path_err": path_err, "spl_pos": spl_pos, "spl_path": spl_path, "spl_val": spl_val}


def summary(c: dict) -> str:
    n = len(c["ok"])
    se = c["same_events"]

    def mx(k):
        return c[k][se].max() if se.any() else 0.0

    def over(k, tol):
        return int((se & (c[k] > tol)).sum())

    return (f"{c['ok_geom'].sum()}/{n} photons within the position, direction and path bounds, "
            f"{c['ok'].sum()}/{n} also within the splat-value bound; events equal {se.sum()}/{n}; "
            f"max pos {mx('pos_err'):.3g} m, max dir {mx('dir_err'):.3g} rad, max path {mx('path_err'):.3g} m, "
            f"max splat pos {mx('spl_pos'):.3g} m, max splat path {mx('spl_path'):.3g} m, "
            f"max splat rel value {c['spl_val'].max():.3g}; over the bounds: pos {over('pos_err', POS_TOL_M)}, "
            f"dir {over('dir_err', DIR_TOL_RAD)}, path {over('path_err', PATH_TOL_M)}, splat pos "
            f"{over('spl_pos', POS_TOL_M)}, splat path {over('spl_path', PATH_TOL_M)}, splat value "
            f"{over('spl_val', VALUE_RTOL)}")


def run_pair(setup, n, per_photon=256, weight=1_000_000, threads=0, real_bits=32):
    """The GPU (through the C ABI) and the oracle on the same injected SFMT streams: photon i draws
    from SFMT-19937 seeded with setup.seed + i, the reference's per-photon seeding (photon.cpp:313).
    Returns (gpu records, gpu film, oracle records, oracle film)."""
    import oracle_bridge as ob
    import simpler_b200 as sb
    u, off = ob.sfmt_streams(setup.seed, 0, n, per_photon)
    g, gimg = sb.trace_photons(setup, 0, n, weight, uniforms=u, offsets=off)
    g = sb.records_to_arrays(g)
    r, rimg = ob.oracle_trace(setup, 0, n, weight, uniforms=u, offsets=off, threads=threads, real_bits=real_bits)
    return g, gimg, r, rimg


def accept(g, r, min_ok=0.98, min_events=0.995, min_geom=0.98, min_end=0.995, min_short=0.995) -> dict:
    """compare_records(g, r) and the acceptance bounds of `check`; prints and returns the comparison."""
    n = len(r)
    c = compare_records(g, r)
    end_ok = c["same_events"] & (c["pos_err"] <= POS_TOL_M) & (c["dir_err"] <= DIR_TOL_RAD) & (c["path_err"] <= PATH_TOL_M)
    short = r["er_steps"] <= np.median(r["er_steps"])
    c["end_ok"] = end_ok
    c["short_ok_frac"] = float(c["ok_geom"][short].mean())
    msg = (summary(c) + f"; ends within the bounds {end_ok.sum()}/{n}; photons with at most the median "
           f"{int(np.median(r['er_steps']))} ER steps within the bounds {c['ok_geom'][short].sum()}/{short.sum()}")
    print(msg)
    assert c["same_events"].mean() >= min_events, msg
    assert end_ok.mean() >= min_end, msg
    assert c["short_ok_frac"] >= min_short, msg
    assert c["ok_geom"].mean() >= min_geom, msg
    assert c["ok"].mean() >= min_ok, msg
    return c


def check(setup, n, min_ok=0.98, min_events=0.995, per_photon=256, img_tol=5e-4, real_bits=32, threads=0,
          min_geom=0.98, min_end=0.995, min_short=0.995):
    """Photon-by-photon parity of the GPU against the oracle.

    * at least `min_events` of the photons take the same discrete events;
    * at least `min_end` end within the position, direction and path bounds;
    * at least `min_geom` are within them at every splat too, and at least `min_ok` within every
      bound including the splat values;
    * at least `min_short` of the photons with no more ER steps than the median are within the
      position, direction and path bounds everywhere. The photons outside those bounds are the
      ones whose splats follow long internally reflected connections (tens of thousands of ER
      steps), where the two float march orders (the GPU's reciprocal and fused multiply-adds, the
      reference's h d / n) drift apart by up to micrometres; this bound keeps a defect on ordinary
      paths from hiding among them.

    The films agree to `img_tol` in relative L1. Prints and returns the comparison."""
    g, gimg, r, rimg = run_pair(setup, n, per_photon, real_bits=real_bits, threads=threads)
    assert not (r["end"] == 8).any(), "oracle ran out of injected uniforms"
    c = accept(g, r, min_ok=min_ok, min_events=min_events, min_geom=min_geom, min_end=min_end, min_short=min_short)
    denom = np.abs(rimg).sum()
    if denom > 0:
        rel = np.abs(gimg - rimg).sum() / denom
        assert rel < img_tol, (rel, msg)
    c["film_rel_l1"] = float(np.abs(gimg - rimg).sum() / denom) if denom > 0 else 0.0
    return c
