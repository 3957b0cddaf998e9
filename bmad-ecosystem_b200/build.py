"""Build libbgt.so (sm_100a) in-tree: bmad-ecosystem_b200/bgt/libbgt.so.

    python bmad-ecosystem_b200/build.py [--fmad]

--fmad lets nvcc contract a*b+c into FMA (off by default: the reference's
gfortran -O2 x86-64 build never contracts, and parity is checked against
that operation order).
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRCS = [HERE / "csrc" / "bgt_track.cu", HERE / "csrc" / "bgt_mlp.cu"]
# the tracking kernel's instances, one compilation per group (bgt_track_kernels.cu)
KERNEL_SRC = HERE / "csrc" / "bgt_track_kernels.cu"
N_KERNEL_GROUPS = 10
OUT = HERE / "bgt" / "libbgt.so"


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or Path(c).exists()):
            return c
    return "nvcc"


def build(fmad: bool = False, out: Path = OUT, verbose: bool = False) -> Path:
    deps = list((HERE / "csrc").glob("*")) + list((HERE.parent / "include").glob("*.h"))
    if out.exists() and all(out.stat().st_mtime >= d.stat().st_mtime for d in deps) and not os.environ.get(
            "BGT_FORCE_BUILD"):
        return out
    common = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              f"--fmad={'true' if fmad else 'false'}", "-Xcompiler", "-fPIC"]
    if verbose:
        common.insert(1, "-Xptxas=-v")
    objdir = out.parent / "_obj"
    objdir.mkdir(exist_ok=True)
    jobs = [([], s, objdir / (s.stem + ".o")) for s in SRCS]
    jobs += [([f"-DBGT_KERNEL_GROUP={g}"], KERNEL_SRC, objdir / f"{KERNEL_SRC.stem}_{g}.o")
             for g in range(N_KERNEL_GROUPS)]
    objs = [o for _, _, o in jobs]
    procs = [subprocess.Popen(common + d + ["-c", "-o", str(o), str(s)], stdout=subprocess.PIPE,
                              stderr=subprocess.PIPE, text=True) for d, s, o in jobs]
    errs = []
    for p in procs:
        so, se = p.communicate()
        if p.returncode != 0:
            errs.append(so + se)
        elif verbose:
            sys.stderr.write(se)
    if errs:
        sys.stderr.write("\n".join(errs))
        raise RuntimeError("nvcc failed building libbgt.so")
    r = subprocess.run([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(out)] +
                       [str(o) for o in objs] + ["-lquadmath"], capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libbgt.so")
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--fmad", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.fmad, verbose=a.verbose))
