"""Builds liblddmm_b200.so in-tree with nvcc for sm_100a.

    python -m registration_b200.build [--verbose-ptxas]

Each .cu under registration_b200/csrc is compiled to an object (in parallel)
and linked into registration_b200/liblddmm_b200.so.  Objects are rebuilt only
when a source or header is newer.  The issue-rate probe kernels that the
benchmark measures its peaks with (registration_b200/probe/probe.cu) are a
measurement utility, built into their own registration_b200/probe/liblddmm_probe.so.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblddmm_b200.so")
PROBE_SRC = os.path.join(HERE, "probe", "probe.cu")
PROBE_LIB = os.path.join(HERE, "probe", "liblddmm_probe.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]
HOSTCC = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else None


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0)


def _compile(src, verbose_ptxas):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _newest_header()):
        return obj, ""
    cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
    if HOSTCC:
        cmd += ["-ccbin", HOSTCC]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    return obj, r.stderr


def build(verbose_ptxas=False, jobs=None):
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    logs = []
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    objs = [o for o, _ in results]
    logs = [l for _, l in results if l]
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if HOSTCC:
            cmd += ["-ccbin", HOSTCC]
        subprocess.run(cmd, check=True)
    build_probe()
    return LIB, logs


def build_probe():
    if os.path.exists(PROBE_LIB) and os.path.getmtime(PROBE_LIB) >= os.path.getmtime(PROBE_SRC):
        return PROBE_LIB
    cmd = [NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler",
                           "-fvisibility=hidden", "-shared", PROBE_SRC, "-o", PROBE_LIB, "-lcudart"]
    if HOSTCC:
        cmd += ["-ccbin", HOSTCC]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (PROBE_SRC, r.stdout, r.stderr))
    return PROBE_LIB


if __name__ == "__main__":
    lib, logs = build(verbose_ptxas="--verbose-ptxas" in sys.argv)
    for l in logs:
        print(l)
    print(lib)
