"""Build the icarion_b200 CUDA library in-tree for sm_100a.

    python -m icarion_b200.build [--force] [--jobs N]

Compiles every ``csrc/*.cu`` translation unit with nvcc
(``-gencode arch=compute_100a,code=sm_100a -lineinfo``) into
``icarion_b200/_lib/libicarion_b200.so``.  Per-unit flags:

* ``icb_step_fp64.cu``, ``icb_step1_fp64.cu``   ``--fmad=false`` (bit-faithful IEEE double push)
* ``icb_step_mixed.cu``, ``icb_step_hilo.cu``, ``icb_step1_mixed.cu``, ``icb_step1_hilo.cu``,
  ``icb_mathcheck.cu``  ``-use_fast_math``

Objects are rebuilt only when a source or header is newer than the object.
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
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIBDIR = PKG / "_lib"
LIB = LIBDIR / "libicarion_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
          "-Xcompiler", "-Wall", "-diag-suppress", "177,550", "-I", str(INCLUDE), "-I", str(CSRC)]
PER_UNIT = {
    "icb_step_fp64.cu": ["--fmad=false"],
    "icb_step_mixed.cu": ["-use_fast_math"],
    "icb_step_hilo.cu": ["-use_fast_math"],
    "icb_step1_fp64.cu": ["--fmad=false"],
    "icb_step1_mixed.cu": ["-use_fast_math"],
    "icb_step1_hilo.cu": ["-use_fast_math"],
    "icb_mathcheck.cu": ["-use_fast_math"],
}
LINK_LIBS = ["-lcufft"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the icarion_b200 CUDA library cannot be built")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def _stale(src: Path, obj: Path, hdr_mtime: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or hdr_mtime > t


def _compile(src: Path, obj: Path, verbose: bool) -> tuple[Path, str]:
    cmd = [nvcc(), *ARCH, *COMMON, *PER_UNIT.get(src.name, []), "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return obj, res.stderr


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    hdr_mtime = max((h.stat().st_mtime for h in _headers()), default=0.0)
    todo = [(s, OBJ / (s.stem + ".o")) for s in srcs]
    stale = [(s, o) for s, o in todo if force or _stale(s, o, hdr_mtime)]
    if stale:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
            for obj, log in ex.map(lambda so: _compile(so[0], so[1], verbose), stale):
                if verbose and log:
                    print(f"--- {obj.name}\n{log}", file=sys.stderr)
    objs = [o for _, o in todo]
    if force or stale or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(tmp), *map(str, objs),
               "-L/usr/local/cuda/lib64", *LINK_LIBS, "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIB)
    return LIB


def unit_headers(unit: str) -> list[Path]:
    """The repository headers a translation unit includes, transitively
    (quoted includes resolved in csrc/ and include/)."""
    import re
    seen: dict[str, Path] = {}
    todo = [CSRC / unit]
    while todo:
        f = todo.pop()
        for name in re.findall(r'^\s*#\s*include\s+"([^"]+)"', f.read_text(), re.M):
            for d in (CSRC, INCLUDE):
                p = d / name
                if p.exists() and name not in seen:
                    seen[name] = p
                    todo.append(p)
                    break
    return [seen[k] for k in sorted(seen)]


def kernel_source_hash(unit: str = "icb_step_mixed.cu") -> str:
    """sha256 over one translation unit, the headers it includes and its
    nvcc flags: a profile taken of a kernel records this, and readers of the
    profile's figures compare it with the current sources."""
    import hashlib
    h = hashlib.sha256()
    for f in [CSRC / unit] + unit_headers(unit):
        h.update(f.name.encode())
        h.update(f.read_bytes())
    h.update(" ".join(ARCH + COMMON[:4] + PER_UNIT.get(unit, [])).encode())
    return h.hexdigest()


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true", help="print ptxas register/spill info")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose))


if __name__ == "__main__":
    main()
