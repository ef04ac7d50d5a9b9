"""Build the CUDA library libwildfires_b200.so in-tree for sm_100a.

Every .cu/.cpp file under csrc/ is compiled by nvcc into an object under
_build/ (rebuilt when the file or any header is newer), then linked into
wildfires_b200/libwildfires_b200.so with the static CUDA runtime.  The ptxas
resource report of every kernel is written to _build/<source>.ptxas.log.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libwildfires_b200.so")
DROPIN = os.path.join(HERE, "libwildfires_b200_dropin.a")
NVCC = os.environ.get("WF_NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-I" + os.path.join(ROOT, "include"),
          "-ccbin", "/usr/bin/g++"]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    inc = os.path.join(ROOT, "include")
    hs += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return hs


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    hdr_mtime = max(os.path.getmtime(h) for h in _headers())
    objs = []
    for src in _sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime):
            continue
        cmd = [NVCC] + ARCH + COMMON + ["-Xptxas", "-v", "-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [NVCC] + COMMON + ["-x", "c++", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        with open(os.path.join(BUILD, os.path.basename(src) + ".ptxas.log"), "w") as f:
            f.write(r.stdout + r.stderr)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed on %s" % src)
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-ccbin", "/usr/bin/g++"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    _build_dropin(verbose, force)
    return LIB


def _build_dropin(verbose=False, force=False):
    """libwildfires_b200_dropin.a: the reference's C++ solver entry points
    (include/wf_dropin.h) for programs that link the reference's other objects."""
    src = os.path.join(HERE, "dropin", "dropin.cu")
    obj = os.path.join(BUILD, "dropin.o")
    hdr_mtime = max(os.path.getmtime(h) for h in _headers())
    if not force and os.path.exists(DROPIN) and os.path.getmtime(DROPIN) >= max(os.path.getmtime(src), hdr_mtime):
        return DROPIN
    cmd = [NVCC] + COMMON + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed on %s" % src)
    if os.path.exists(DROPIN):
        os.remove(DROPIN)
    r = subprocess.run(["ar", "rcs", DROPIN, obj], capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("ar failed")
    return DROPIN


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
