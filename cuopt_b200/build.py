"""Build recipe for libcuopt_b200.so (the C-ABI library) — sm_100a only.

Each translation unit under csrc/ is compiled by nvcc for ``-gencode arch=compute_100a,code=sm_100a``
in parallel, then linked into ``cuopt_b200/libcuopt_b200.so`` with a static CUDA runtime so the
library has no run-time dependency beyond the driver.  Usage::

    python -m cuopt_b200.build          # incremental
    python -m cuopt_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build"
LIB = PKG / "libcuopt_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    # The system compiler; some images put a wrapper first on PATH that lacks libgomp specs.
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else (shutil.which("g++") or "g++")


def _flags() -> list[str]:
    return [
        "-O3", "-lineinfo", "-std=c++17", *ARCH,
        "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
        "-ccbin", _host_cxx(), f"-I{ROOT / 'include'}", f"-I{CSRC}",
    ]


def _sources() -> list[Path]:
    return sorted([*CSRC.glob("*.cu"), *CSRC.glob("*.cpp")])


def _headers_mtime() -> float:
    hs = [*CSRC.glob("*.cuh"), *CSRC.glob("*.hpp"), *CSRC.glob("*.h"), *(ROOT / "include").rglob("*.h")]
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, force: bool, hdr_mtime: float, verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_mtime):
        return obj
    lang = ["-x", "cu"] if src.suffix == ".cu" else ["-x", "c++"]
    cmd = [_nvcc(), *lang, *_flags(), "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    hdr = _headers_mtime()
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, hdr, verbose), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [_nvcc(), *ARCH, "-shared", "-cudart", "static", "-ccbin", _host_cxx(),
               "-Xcompiler", "-fPIC", "-o", str(LIB), *map(str, objs), "-lpthread", "-ldl"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/spill usage")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
