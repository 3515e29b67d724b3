"""Python entry points over the C ABI: render, plans, parity traces and field probes."""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _lib as L
from .scene import Setup


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def render(setup: Setup, n_photons: int) -> tuple[np.ndarray, L.Stats]:
    """One-shot render (the reference's Renderer::renderImage). Returns the film as a
    (z, y, x) float64 array -- index z*X*Y + y*X + x, the reference's Image3 layout -- and stats."""
    lib = L.load()
    sc, md, fd, op = setup.descs()
    img = np.zeros(setup.film_shape(), dtype=np.float64)
    st = L.Stats()
    L.check(lib.smp_render(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), int(n_photons), _ptr(img), C.byref(st)))
    return img, st


class Plan:
    """Device-resident scene + film; repeated renders pay no setup."""

    def __init__(self, setup: Setup):
        self.setup = setup
        self.lib = L.load()
        self._descs = setup.descs()
        sc, md, fd, op = self._descs
        h = C.c_void_p()
        L.check(self.lib.smp_plan_create(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), C.byref(h)))
        self.handle = h

    def clear(self, stream: int = 0) -> None:
        L.check(self.lib.smp_plan_clear(self.handle, C.c_void_p(stream)))

    def trace(self, first: int, n: int, weight_photons: int, stream: int = 0) -> None:
        L.check(self.lib.smp_plan_trace(self.handle, int(first), int(n), int(weight_photons), C.c_void_p(stream)))

    def read_image(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.zeros(self.setup.film_shape(), dtype=np.float64)
        L.check(self.lib.smp_plan_read_image(self.handle, _ptr(out), 0, None))
        return out

    def read_image_device(self, dev_ptr: int, stream: int = 0) -> None:
        L.check(self.lib.smp_plan_read_image(self.handle, C.c_void_p(dev_ptr), 1, C.c_void_p(stream)))

    def film(self) -> tuple[int, int]:
        p = C.c_void_p()
        b = C.c_int32()
        L.check(self.lib.smp_plan_film(self.handle, C.byref(p), C.byref(b)))
        return p.value, b.value

    def stats(self) -> L.Stats:
        st = L.Stats()
        L.check(self.lib.smp_plan_stats(self.handle, C.byref(st)))
        return st

    def render(self, n_photons: int) -> tuple[np.ndarray, L.Stats]:
        img = np.zeros(self.setup.film_shape(), dtype=np.float64)
        st = L.Stats()
        L.check(self.lib.smp_plan_render(self.handle, int(n_photons), _ptr(img), C.byref(st)))
        return img, st

    def adjoint(self, dJ_dfilm: np.ndarray, first: int = 0, n: int | None = None,
                weight_photons: int | None = None) -> tuple[np.ndarray, L.AdjointStats]:
        """Gradient of J = sum(dJ_dfilm * film) over the field parameters (`field_params` order)
        for the film of photons [first, first + n) of this plan's render (weight_photons as in
        `trace`; each defaults to the other)."""
        g = np.ascontiguousarray(dJ_dfilm, dtype=np.float64)
        if g.shape != self.setup.film_shape():
            raise ValueError(f"dJ_dfilm shape {g.shape} != film {self.setup.film_shape()}")
        if n is None and weight_photons is None:
            raise ValueError("give n or weight_photons")
        n = int(n if n is not None else weight_photons)
        w = int(weight_photons if weight_photons is not None else n)
        grad = np.zeros(param_count(self.setup), dtype=np.float64)
        st = L.AdjointStats()
        L.check(self.lib.smp_plan_adjoint(self.handle, int(first), n, w, _ptr(g), _ptr(grad), C.byref(st)))
        return grad, st

    def tune(self, n_sample: int) -> L.Tuning:
        """Autotune the slot pool (march-kernel block size, slots per lane, chunk) with trial traces of
        n_sample photons; cached per process for the same configuration. Clears the film."""
        t = L.Tuning()
        L.check(self.lib.smp_plan_tune(self.handle, int(n_sample), C.byref(t)))
        return t

    def tune_step(self, n_sample: int, rmse_budget: float) -> tuple[float, float]:
        """The step-size autotuner (smp_plan_tune_step): sets the plan's ER step to the largest
        multiple (2 .. 32, capped by the field's shortest length scale) of the field's own step whose
        film on photons [0, n_sample) stays within `rmse_budget` relative RMSE of the film at the own
        step (searched in the mixed form; an FP32 plan uses a mixed-form copy of itself, except a
        spline plan). Returns (step in metres, measured RMSE). The film is cleared; set_field
        restores the field's own step."""
        step, rmse = C.c_double(), C.c_double()
        L.check(self.lib.smp_plan_tune_step(self.handle, int(n_sample), float(rmse_budget), C.byref(step),
                                            C.byref(rmse)))
        return step.value, rmse.value

    def set_field(self, setup: Setup) -> None:
        fd = setup.field_desc()
        L.check(self.lib.smp_plan_set_field(self.handle, C.byref(fd)))
        self._fd_keep = fd

    def close(self) -> None:
        if self.handle:
            self.lib.smp_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _instance_descs(setup: Setup, instances: list):
    import dataclasses
    n = len(instances)
    arr = (L.InstanceDesc * n)()
    for i, inst in enumerate(instances):
        over = {k: v for k, v in inst.items() if k not in ("n_photons", "seed")}
        s = dataclasses.replace(setup, **over)
        arr[i].field = s.field_desc()
        arr[i].medium = s.medium_desc()
        arr[i].n_photons = int(inst["n_photons"])
        arr[i].seed = int(inst.get("seed", 0))
    return arr


def render_batch(setup: Setup, instances: list) -> tuple[np.ndarray, L.Stats]:
    """A sweep of many field / medium configurations over one scene, in one slot pool.

    `instances` is a list of dicts: any Setup field or medium attribute to override
    (mode, n_max, n_clip, f_u, speed_u, phi_min, phi_max, sigma_t, albedo, g, er_stepsize, ...)
    plus `n_photons` and `seed`. Returns the films as an (n_inst, z, y, x) float64 array and the
    statistics of the whole sweep. Photon j of instance i draws the stream (seed_i, j), so each
    film equals a single render of that configuration with that seed."""
    lib = L.load()
    n = len(instances)
    arr = _instance_descs(setup, instances)
    sc, _, _, op = setup.descs()
    films = np.zeros((n,) + setup.film_shape(), dtype=np.float64)
    st = L.Stats()
    L.check(lib.smp_render_batch(C.byref(sc), arr, n, C.byref(op), _ptr(films), C.byref(st)))
    return films, st


def tune_batch_steps(setup: Setup, instances: list, rmse_budget: float, n_sample: int = 20000):
    """The step-size autotuner of a batched sweep (smp_batch_tune_steps): per instance, the largest
    multiple (2 .. 32, at most an eighth of the ultrasound wavelength) of its ER step whose film on
    its first n_sample photons stays within `rmse_budget` relative RMSE of the film at its own step,
    on the same photons (largest allowed multiple first, then bisection; the search renders in the
    mixed form, and an instance that misses at every multiple searches again with 10 n_sample
    photons). Returns (steps, rmse, rounds); pass {"er_stepsize": steps[i]} into instance i for
    render_batch."""
    lib = L.load()
    n = len(instances)
    arr = _instance_descs(setup, instances)
    sc, _, _, op = setup.descs()
    steps = np.zeros(n)
    rmse = np.zeros(n)
    rounds = C.c_int32(0)
    L.check(lib.smp_batch_tune_steps(C.byref(sc), arr, n, C.byref(op), int(n_sample), float(rmse_budget),
                                     _ptr(steps), _ptr(rmse), C.byref(rounds)))
    return steps, rmse, int(rounds.value)


def trace_photons(setup: Setup, first: int, n: int, weight_photons: int,
                  uniforms: np.ndarray | None = None, offsets: np.ndarray | None = None,
                  with_image: bool = True):
    """Parity mode: per-photon records (and the film) for photons [first, first+n)."""
    lib = L.load()
    sc, md, fd, op = setup.descs()
    recs = (L.PhotonRecord * n)()
    img = np.zeros(setup.film_shape(), dtype=np.float64) if with_image else None
    u = o = None
    if uniforms is not None:
        u = np.ascontiguousarray(uniforms, dtype=np.float32)
        o = np.ascontiguousarray(offsets, dtype=np.int64)
    rc = lib.smp_trace_photons(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), int(first), int(n),
                               int(weight_photons), _ptr(u) if u is not None else None,
                               _ptr(o) if o is not None else None, recs, _ptr(img) if img is not None else None)
    L.check(rc)
    return recs, img


def field_eval(setup: Setup, scaling: float, points: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """n and grad n at points (N,3) with the march kernel's own field code."""
    lib = L.load()
    fd = setup.field_desc()
    pts = np.ascontiguousarray(points, dtype=np.float64)
    n = np.zeros(len(pts))
    g = np.zeros((len(pts), 3))
    L.check(lib.smp_field_eval(C.byref(fd), float(scaling), len(pts), _ptr(pts), _ptr(n), _ptr(g)))
    return n, g


def records_to_arrays(recs) -> dict:
    """Flatten PhotonRecords into numpy arrays for comparisons."""
    n = len(recs)
    raw = np.ctypeslib.as_array(C.cast(recs, C.POINTER(C.c_uint8)), shape=(n * C.sizeof(L.PhotonRecord),))
    dt = np.dtype([
        ("photon", "<i8"), ("end", "<i4"), ("draws", "<i4"), ("depth", "<i4"), ("n_splats", "<i4"),
        ("pos", "<f4", 3), ("dir", "<f4", 3), ("total_optical", "<f8"), ("er_steps", "<i8"),
        ("splats", [("p", "<f4", 3), ("depth", "<i4"), ("pathlength", "<f8"), ("value", "<f8")], L.SMP_TRACE_MAX_SPLATS),
    ])
    assert dt.itemsize == C.sizeof(L.PhotonRecord), (dt.itemsize, C.sizeof(L.PhotonRecord))
    return raw.view(dt).copy()


# ---- field parameters of the adjoint -------------------------------------------------------------
def param_count(setup: Setup) -> int:
    """Length of the parameter vector `adjoint` differentiates (Bessel: n_max, phi_min, phi_max;
    plane waves: amplitudes then phases; spline: the coefficient grid, x fastest)."""
    fd = setup.field_desc()
    n = L.load().smp_adjoint_param_count(C.byref(fd))
    if n < 0:
        L.check(int(n))
    return int(n)


def field_params(setup: Setup) -> np.ndarray:
    """The setup's differentiable field parameters as one float64 vector."""
    if setup.field_type == L.FIELD_PLANEWAVE:
        return np.concatenate([np.asarray(setup.wave_amp, np.float64), np.asarray(setup.wave_phase, np.float64)])
    if setup.field_type == L.FIELD_SPLINE:
        return np.asarray(setup.grid_coeff, np.float64).ravel().copy()
    if setup.field_type == L.FIELD_BESSEL:
        return np.array([setup.n_max, setup.phi_min, setup.phi_max], dtype=np.float64)
    raise ValueError("the adjoint is built for Bessel, plane-wave and spline fields")


def with_field_params(setup: Setup, theta) -> Setup:
    """A copy of `setup` with its field parameters replaced by `theta` (`field_params` order)."""
    theta = np.asarray(theta, dtype=np.float64)
    if setup.field_type == L.FIELD_PLANEWAVE:
        w = len(setup.wave_amp)
        return dataclasses.replace(setup, wave_amp=tuple(float(x) for x in theta[:w]),
                                   wave_phase=tuple(float(x) for x in theta[w:2 * w]))
    if setup.field_type == L.FIELD_SPLINE:
        return dataclasses.replace(setup, grid_coeff=theta.reshape(np.shape(setup.grid_coeff)).astype(np.float32))
    if setup.field_type == L.FIELD_BESSEL:
        return dataclasses.replace(setup, n_max=float(theta[0]), phi_min=float(theta[1]), phi_max=float(theta[2]))
    raise ValueError("the adjoint is built for Bessel, plane-wave and spline fields")


def roi_weights(setup: Setup, size: int = 32) -> np.ndarray:
    """dJ/dfilm of the throughput of a central size x size pixel region, summed over all bins."""
    g = np.zeros(setup.film_shape(), dtype=np.float64)
    z, y, x = g.shape
    y0, x0 = (y - size) // 2, (x - size) // 2
    g[:, y0:y0 + size, x0:x0 + size] = 1.0
    return g


def shard_range(n_photons: int, rank: int, world: int) -> tuple[int, int]:
    """This rank's contiguous photon range [first, first + n) of an n_photons render split over
    `world` processes. Photon k draws Philox stream (seed, k) on any rank, so the shards add up to
    the single-process render for any world size."""
    per = -(-int(n_photons) // int(world))
    first = int(rank) * per
    return first, max(0, min(per, int(n_photons) - first))


_COUNT_KEYS = ("photons", "er_steps", "splats", "step_cap_hits", "nan_photons")
_ADJ_COUNT_KEYS = ("photons", "dropped", "skipped", "aborted", "replay_mismatch")


def render_sharded(plan, n_photons: int, rank: int = 0, world: int = 1, all_reduce=None,
                   stream: int = 0) -> tuple[np.ndarray, dict]:
    """The film of the n_photons render over `world` processes (one GPU each, photons split by
    contiguous index range): this rank clears its plan's film, traces its own photon range with the render's
    photon weight (Li T / n_photons, photon.h:76-80), and reads the FP64 film back; `all_reduce` (a
    callable that sums a float64 numpy array over the ranks and returns it, e.g. over
    torch.distributed) combines the films and the photon / step / splat counts in one call. Returns
    (film, counts); without all_reduce, this rank's share."""
    first, n = shard_range(n_photons, rank, world)
    plan.clear(stream)
    if n > 0:
        plan.trace(first, n, int(n_photons), stream)
    film = plan.read_image()
    st = plan.stats()
    counts = np.array([float(getattr(st, k)) for k in _COUNT_KEYS])
    if all_reduce is not None:
        packed = all_reduce(np.concatenate([film.ravel(), counts]))
        film = np.asarray(packed[:film.size]).reshape(film.shape)
        counts = np.asarray(packed[film.size:])
    return film, {k: int(round(v)) for k, v in zip(_COUNT_KEYS, counts)}


def adjoint_sharded(plan, dJ_dfilm: np.ndarray, n_photons: int, rank: int = 0, world: int = 1,
                    all_reduce=None) -> tuple[np.ndarray, dict]:
    """The gradient of the n_photons render over `world` processes (one GPU each): this rank
    differentiates its contiguous photon range (`shard_range`) and `all_reduce` (a callable that
    sums a float64 array over the ranks and returns it) combines the gradients together with the
    photon counts of the adjoint statistics, so every rank sees how many photons were
    differentiated and how many were dropped, skipped (sensor marches) or aborted anywhere. `plan`
    is this rank's Plan (anything with Plan.adjoint's signature). Returns (gradient, counts)."""
    first, n = shard_range(n_photons, rank, world)
    counts = np.zeros(len(_ADJ_COUNT_KEYS))
    if n > 0:
        grad, st = plan.adjoint(dJ_dfilm, first, n, int(n_photons))
        grad = np.asarray(grad, dtype=np.float64)
        if st is not None:
            counts = np.array([float(getattr(st, k)) for k in _ADJ_COUNT_KEYS])
    else:
        grad = np.zeros(param_count(plan.setup), dtype=np.float64)
    if all_reduce is not None:
        packed = all_reduce(np.concatenate([grad, counts]))
        grad, counts = np.asarray(packed[:grad.size]), np.asarray(packed[grad.size:])
    return grad, {k: int(round(v)) for k, v in zip(_ADJ_COUNT_KEYS, counts)}


def adjoint(setup: Setup, n_photons: int, dJ_dfilm: np.ndarray) -> tuple[np.ndarray, L.AdjointStats]:
    """One-shot gradient of sum(dJ_dfilm * film) for the n_photons render of `setup`."""
    lib = L.load()
    sc, md, fd, op = setup.descs()
    g = np.ascontiguousarray(dJ_dfilm, dtype=np.float64)
    if g.shape != setup.film_shape():
        raise ValueError(f"dJ_dfilm shape {g.shape} != film {setup.film_shape()}")
    grad = np.zeros(param_count(setup), dtype=np.float64)
    st = L.AdjointStats()
    L.check(lib.smp_render_adjoint(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), int(n_photons), _ptr(g),
                                   _ptr(grad), C.byref(st)))
    return grad, st


# ---- static fields as a tricubic grid ---------------------------------------------------------
def sources_to_spline(setup: Setup, n: int = 96, margin: int = 6) -> Setup:
    """The point-source field of `setup` sampled on an n^3 grid of nodes (with the march's own field
    code, on the GPU), prefiltered into tricubic B-spline coefficients (smp_spline_prefilter, the
    reference's Spline<3>::build3d), returned as a spline-field setup: the reference's
    rif_interpolated route for a field that is fixed in time. Every evaluation then reads 64
    coefficients instead of summing every point source (1e5 for the reference's arcs). The grid
    reaches `margin` node spacings beyond the medium box on every side, because the prefilter's
    mirror boundary flattens the field's normal derivative over the last few nodes. The gaps stay
    those of `setup`. For the reference's default arcs (1 MHz-scale wavelengths of 1.8 mm in a
    10 mm box) a 96^3 grid reproduces grad n to 7e-4 and a 128^3 grid to 3e-4 of its largest value;
    n to the float resolution of n itself."""
    if setup.field_type != L.FIELD_SOURCES:
        raise ValueError("sources_to_spline takes a point-source setup")
    lo = np.asarray(setup.medium_l, dtype=np.float64)
    hi = np.asarray(setup.medium_r, dtype=np.float64)
    h = (hi - lo) / (n - 1 - 2 * margin)
    lo, hi = lo - margin * h, hi + margin * h
    axes = [np.linspace(lo[i], hi[i], n) for i in range(3)]
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    pts = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    # dn = n - n_o at the nodes (n_o = 0 keeps dn's own float precision), no gating at the nodes
    probe = dataclasses.replace(setup, n_o=0.0, emitter_gap=-1e-3, sensor_gap=-1e-3)
    vals, _ = field_eval(probe, 0.0, pts)
    samples = np.ascontiguousarray(vals.reshape(n, n, n), dtype=np.float32)
    coeff = np.zeros_like(samples)
    dims = np.array([n, n, n], dtype=np.int32)
    L.check(L.load().smp_spline_prefilter(_ptr(samples), _ptr(dims), _ptr(coeff)))
    return dataclasses.replace(setup, field_type=L.FIELD_SPLINE, grid_coeff=coeff, grid_offset=float(setup.n_o),
                               grid_min=tuple(float(v) for v in lo), grid_max=tuple(float(v) for v in hi))
