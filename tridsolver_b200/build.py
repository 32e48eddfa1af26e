"""Build the tridsolver_b200 shared libraries in-tree with nvcc (sm_100a).

    python -m tridsolver_b200.build          # or tridsolver_b200.build.build()

Outputs (next to this file, git-ignored, travel with the repository):
    libtridb200.so             scalar C ABI (9-argument strided batch), block,
                               adjoint, varlen, ADI entry points
    libtridb200_cudacompat.so  the same with the reference GPU library's
                               11-argument strided-batch signatures
Objects go to tridsolver_b200/_build/.
"""

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xptxas", "-warn-spills", "--expt-relaxed-constexpr",
                     "-I", os.path.join(ROOT, "include")]

# sources shared by both libraries
COMMON = ["kern_scalar.cu", "kern_xtma.cu", "kern_sptma.cu", "kern_general.cu", "kern_block.cu",
          "kern_varlen.cu", "kern_adi.cu", "kern_xcta.cu", "kern_split.cu", "tma_host.cu"]
MAIN = ["api_scalar.cu", "kern_ext.cu"]
COMPAT = [("api_scalar.cu", ["-DTRID_CUDACOMPAT"]), ("api_compat.cu", [])]

LIBS = {
    "libtridb200.so": [(s, []) for s in COMMON + MAIN],
    "libtridb200_cudacompat.so": [(s, []) for s in COMMON] + COMPAT,
}


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return exe


def _obj_name(src, defs):
    tag = "_".join(d.lstrip("-D").lower() for d in defs)
    base = os.path.splitext(src)[0]
    return os.path.join(BUILD, base + ("_" + tag if tag else "") + ".o")


def _compile(src, defs, verbose):
    obj = _obj_name(src, defs)
    srcp = os.path.join(CSRC, src)
    deps = [srcp] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(p) for p in deps):
        return obj
    cmd = [nvcc()] + NVCC_FLAGS + defs + ["-c", srcp, "-o", obj]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)
    return obj


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    jobs = {(s, tuple(d)) for objs in LIBS.values() for s, d in objs}
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        futs = {ex.submit(_compile, s, list(d), verbose): (s, d) for s, d in jobs}
        for f in cf.as_completed(futs):
            f.result()
    for lib, objs in LIBS.items():
        out = os.path.join(HERE, lib)
        obj_paths = [_obj_name(s, d) for s, d in objs]
        # the object list of the last link: a changed list relinks too
        stamp = os.path.join(BUILD, lib + ".objs")
        listed = "\n".join(obj_paths)
        same = os.path.exists(stamp) and open(stamp).read() == listed
        if same and os.path.exists(out) and \
                os.path.getmtime(out) >= max(os.path.getmtime(o) for o in obj_paths):
            continue
        cmd = [nvcc()] + ARCH + ["-shared", "-o", out] + obj_paths
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed for {lib}:\n{r.stdout}\n{r.stderr}")
        with open(stamp, "w") as f:
            f.write(listed)
    return [os.path.join(HERE, lib) for lib in LIBS]


if __name__ == "__main__":
    for p in build(verbose="-v" in sys.argv):
        print(p)
