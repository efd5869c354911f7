"""Build the CUDA library libtsb200.so (sm_100a) in-tree.

    python -m trottersuzuki_b200.build          (from trotter-suzuki-mpi_b200/)

Each .cu under csrc/ is compiled to an object under _build/ in parallel, then
linked next to this file so that the package loads it from its own folder.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
REPO = os.path.dirname(PKG_ROOT)
CSRC = os.path.join(PKG_ROOT, "csrc")
INCLUDE = os.path.join(REPO, "include")
BUILD = os.path.join(REPO, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC]


def _nccl_include():
    """nccl.h (types only: the library is loaded at run time): the NCCL
    wheel's, else the system's."""
    try:
        import nvidia.nccl
        d = os.path.join(list(nvidia.nccl.__path__)[0], "include")
        if os.path.exists(os.path.join(d, "nccl.h")):
            return d
    except ImportError:
        pass
    return "/usr/include"


FLAGS.append("-I" + _nccl_include())


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _includes(path, seen=None):
    """Files under csrc/ and include/ that `path` includes, recursively."""
    seen = set() if seen is None else seen
    try:
        text = open(path).read()
    except OSError:
        return seen
    for line in text.splitlines():
        line = line.strip()
        if line.startswith("#include \""):
            name = line.split('"')[1]
            for d in (CSRC, INCLUDE):
                f = os.path.join(d, name)
                if os.path.exists(f) and f not in seen:
                    seen.add(f)
                    _includes(f, seen)
    return seen


def _compile(src, extra):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    deps = [src] + sorted(_includes(src))
    if _stale(obj, deps):
        # the object carries the sources' time at the start of the compile,
        # so that an edit made while it compiles leaves it stale
        stamp = max(os.path.getmtime(d) for d in deps)
        cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", src, "-o", obj + ".tmp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        os.replace(obj + ".tmp", obj)
        os.utime(obj, (stamp, stamp))
    return obj


HOST = os.path.join(PKG_ROOT, "host")
CXX = os.environ.get("TS_B200_CXX", "g++")


def build_host(verbose=True):
    """The C++ host layer (drop-in API) linked against libtsb200.so."""
    srcs = sorted(os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".cpp"))
    deps = srcs + [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".h")]
    deps += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    out = os.path.join(HERE, "libtrottersuzuki_b200.so")
    cuda_lib = os.path.join(HERE, "libtsb200.so")
    if _stale(out, deps + [cuda_lib]):
        cmd = [CXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
               "-I" + INCLUDE, "-I" + HOST] + srcs + [
            "-L" + HERE, "-ltsb200", "-Wl,-rpath,$ORIGIN", "-o", out + ".tmp"]
        subprocess.check_call(cmd)
        os.replace(out + ".tmp", out)
    if verbose:
        print("built", out)
    return out


def build(verbose=True, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, list(extra)), srcs))
    out = os.path.join(HERE, "libtsb200.so")
    if _stale(out, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", out + ".tmp"] + objs + ["-lcudart", "-ldl"]
        subprocess.check_call(cmd)
        os.replace(out + ".tmp", out)
    if verbose:
        print("built", out)
    build_host(verbose)
    return out


if __name__ == "__main__":
    build(extra=sys.argv[1:])
