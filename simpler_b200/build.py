"""Build the native parts of simpler_b200 in-tree.

* ``libsimpler_b200.so`` -- the CUDA kernels and the C ABI (``include/simpler_b200.h``),
  compiled for sm_100a only, plus the C++ host layer (``csrc/host/smp_host.cpp``: file formats,
  the reference's key=value and JSON front-ends);
* ``bin/renderer3d`` and ``bin/simplER`` -- the reference's two command-line front-ends over it;
* ``pybind_ext/{tvector,phase,medium,image,scene,photon}_pybind`` -- the reference's Python modules,
  compiled with pybind11 over the C ABI;
* the CPU oracle (``oracle/liboracle*.so``) and, when the reference checkout is present, the
  reference's own primitives (``oracle/_ref``) -- test infrastructure, built here so the GPU box
  receives them prebuilt.

Usage: ``python -m simpler_b200.build [--verbose]``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsimpler_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
    # no automatic a*b+c contraction: every kernel (and the CPU oracle) rounds the same expression
    # the same way, so the single-kernel and two-kernel paths give identical photons; the hot
    # arithmetic uses explicit fmaf
    "-fmad=false",
]

# the kernels are split over translation units (dispatch.h) so that they compile in parallel
CU_SOURCES = ["capi.cu", "k_march.cu", "k_wave.cu", "k_adjoint.cu", "adjoint_sweep.cu", "host/smp_host.cpp"]
# Per-file overrides of NVCC_FLAGS. The adjoint's backward sweep does not take part in any
# bit-for-bit comparison (its inputs are read back from the replayed trajectories), so its
# arithmetic may contract a*b+c into FMAs.
FILE_FLAGS = {"adjoint_sweep.cu": ["-fmad=true"]}
HEADERS = ["kparams.h", "dispatch.h", "dev_math.cuh", "dev_field.cuh", "march.cuh", "wavefront.cuh", "plain.cuh",
           "adjoint.cuh", "host/smp_host.h"]
BIN = os.path.join(HERE, "bin")
MAINS = {"renderer3d": "host/renderer3d_main.cpp", "simplER": "host/simpler_main.cpp",
         "merge_renderings": "host/merge_main.cpp"}


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_library(verbose: bool = False, force: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in CU_SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "simpler_b200.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs, procs = [], []
    for f in CU_SOURCES:
        obj = os.path.join(objdir, os.path.basename(f) + ".o")
        flags = [x for x in NVCC_FLAGS if x != "-shared"]
        extra = FILE_FLAGS.get(f, [])
        if any(x.startswith("-fmad") for x in extra):
            flags = [x for x in flags if not x.startswith("-fmad")]
        cmd = [_nvcc(), *flags, *extra, "-c", os.path.join(CSRC, f), "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((f, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        objs.append(obj)
    for f, pr in procs:
        out, err = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError(f"nvcc failed on {f}:\n{out}\n{err}")
        if verbose:
            sys.stderr.write(err)
    res = subprocess.run([_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", LIB + ".tmp"],
                         capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_frontends(force: bool = False) -> None:
    """The command-line front-ends, linked against the library with an rpath to it."""
    os.makedirs(BIN, exist_ok=True)
    cxx = shutil.which("g++") or "g++"
    for name, src in MAINS.items():
        out = os.path.join(BIN, name)
        deps = [os.path.join(CSRC, src), os.path.join(CSRC, "host", "smp_host.h"), LIB]
        if not force and not _stale(out, deps):
            continue
        cmd = [cxx, "-std=c++17", "-O2", os.path.join(CSRC, src), "-I", os.path.join(CSRC, "host"),
               "-L", HERE, "-lsimpler_b200", "-Wl,-rpath,$ORIGIN/..", "-o", out + ".tmp"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"front-end build failed:\n{res.stdout}\n{res.stderr}")
        os.replace(out + ".tmp", out)


PYBIND_DIR = os.path.join(HERE, "pybind_ext")
PYBIND_MODULES = ["tvector_pybind", "phase_pybind", "medium_pybind", "image_pybind", "scene_pybind", "photon_pybind"]


def build_pybind(force: bool = False) -> None:
    """The reference's six pybind11 modules (renderer/pybindFiles/*_pybind.cpp) under their own names,
    compiled over the C ABI into simpler_b200/pybind_ext/ (put that directory on sys.path, as the
    reference's users put its build directory there, and `import scene_pybind` works unchanged)."""
    import sysconfig

    import pybind11
    os.makedirs(PYBIND_DIR, exist_ok=True)
    src_dir = os.path.join(CSRC, "pybind")
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    cxx = shutil.which("g++") or "g++"
    procs = []
    for name in PYBIND_MODULES:
        out = os.path.join(PYBIND_DIR, name + suffix)
        src = os.path.join(src_dir, name + ".cpp")
        deps = [src, os.path.join(src_dir, "pybind_types.h"), os.path.join(CSRC, "host", "smp_host.h"),
                os.path.join(ROOT, "include", "simpler_b200.h"), LIB]
        if not force and not _stale(out, deps):
            continue
        cmd = [cxx, "-std=c++17", "-O2", "-shared", "-fPIC", src, "-I", pybind11.get_include(),
               "-I", sysconfig.get_paths()["include"], "-L", HERE, "-lsimpler_b200", "-Wl,-rpath,$ORIGIN/..",
               "-o", out + ".tmp"]
        procs.append((name, out, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    for name, out, pr in procs:
        o, e = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError(f"pybind module {name} failed to build:\n{o}\n{e}")
        os.replace(out + ".tmp", out)


def build_oracle() -> None:
    """Test infrastructure: the CPU checker and the reference primitives used to pin it."""
    odir = os.path.join(ROOT, "oracle")
    env = dict(os.environ)
    env.pop("CXX", None)
    res = subprocess.run(["make", "-s", "-C", odir, "all"], capture_output=True, text=True, env=env)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    # the recipe finds the reference checkout itself (SIMPLER_REFERENCE_ROOT, else its default
    # location) and does nothing when there is none, as on a machine that only runs prebuilt files
    ref = os.path.join(odir, "ref", "build_ref.sh")
    if os.path.exists(ref):
        res = subprocess.run(["sh", ref], capture_output=True, text=True, env=env)
        if res.returncode != 0:
            raise RuntimeError(f"reference primitives build failed:\n{res.stdout}\n{res.stderr}")


def build_all(verbose: bool = False, force: bool = False) -> None:
    build_library(verbose=verbose, force=force)
    build_frontends(force=force)
    build_pybind(force=force)
    build_oracle()


if __name__ == "__main__":
    build_all(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
