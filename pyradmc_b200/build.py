"""Build the sm_100a shared library of the B200 backend, in-tree.

``python -m pyradmc_b200.build`` compiles each translation unit in ``csrc/``
(``pmc_runtime.cu``, which includes every transport kernel header,
``denoise.cu`` and ``pmc_presolve.cu``) with nvcc for ``sm_100a``, in parallel, and links them into
``_lib/libpmc_b200.so``.  The library is rebuilt only when a source is newer than
it, unless ``force`` is set.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
CSRC = PACKAGE / "csrc"
LIBDIR = PACKAGE / "_lib"
LIBRARY = LIBDIR / "libpmc_b200.so"
INCLUDE = PACKAGE.parent / "include"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    # Approximate float32 transcendentals and division for the float32
    # transport (as the Warp kernels compile with fast_math); the float64
    # reductions use explicit round-to-nearest intrinsics and are unaffected.
    "--use_fast_math",
    "-lineinfo",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC",
]
UNITS = ("pmc_runtime.cu", "denoise.cu", "pmc_presolve.cu")


def nvcc() -> str:
    """Locate nvcc: $CUDA_HOME/bin, /usr/local/cuda/bin, then PATH."""
    for root in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if root and (Path(root) / "bin" / "nvcc").exists():
            return str(Path(root) / "bin" / "nvcc")
    return "nvcc"


def sources() -> list[Path]:
    """Every file the library depends on."""
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def needs_build() -> bool:
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    return any(src.stat().st_mtime > built for src in sources())


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compile the library if it is missing or stale; return its path."""
    if not force and not needs_build():
        return LIBRARY
    LIBDIR.mkdir(exist_ok=True)
    tag = f"tmp{os.getpid()}"
    tmp = LIBRARY.with_suffix(f".so.{tag}")
    objects = [LIBDIR / f"{Path(u).stem}.{tag}.o" for u in UNITS]
    procs = []
    for unit, obj in zip(UNITS, objects):
        cmd = [nvcc(), *ARCH_FLAGS, *NVCC_FLAGS, f"-I{INCLUDE}", "-c", str(CSRC / unit), "-o", str(obj)]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append(subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    failures = []
    for proc in procs:
        out, err = proc.communicate()
        if proc.returncode != 0:
            failures.append(f"nvcc failed ({proc.returncode}):\n{out}\n{err}")
        elif ptxas_info or verbose:
            sys.stderr.write(err)
    try:
        if failures:
            raise RuntimeError("\n".join(failures))
        link = [nvcc(), *ARCH_FLAGS, "-shared", *(str(o) for o in objects), "-lcudart", "-o", str(tmp)]
        proc = subprocess.run(link, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"nvcc link failed ({proc.returncode}):\n{proc.stdout}\n{proc.stderr}")
        tmp.replace(LIBRARY)
    finally:
        tmp.unlink(missing_ok=True)
        for obj in objects:
            obj.unlink(missing_ok=True)
    return LIBRARY


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
