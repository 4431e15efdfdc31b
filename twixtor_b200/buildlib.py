"""Builds the library twixtor_b200/libtwixtor_b200.so with nvcc for sm_100a (in tree).

Strict mode flags: no FMA contraction (-fmad=false), IEEE division and square root, denormals
kept (-ftz=false). The solver's translation units are built a second time for the fast mode. The library is plain C ABI + CUDA runtime; it links no PyTorch.

One generated input: the table of inputs where glibc's logf differs from the library's own
double precision log (csrc/twlog.h), made by running csrc/gen_logf_table.c (it calls this
machine's glibc logf on every positive finite float, a few seconds on all cores) into
_build/logf_table.bin and embedded through csrc/logf_table.S.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtwixtor_b200.so")
SOURCES = ["solver.cu", "fused.cu", "coarse.cu", "image.cu", "smart.cu", "forward.cu", "layers.cu", "filters.cu", "prep.cu", "adjoint.cu", "host_context.cu", "host_solve.cu", "host_compose.cu", "host_layers.cu", "host_clips.cu", "host_time.cu", "host_tune.cu", "host_vecin.cu", "vecin.cu", "debug.cu", "noalloc.cu"]
FAST_SOURCES = ["fused.cu", "solver.cu", "coarse.cu"]  # built a second time for the fast mode
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "-shared", "-cudart", "shared",
]


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "twixtor_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def logf_table_object(verbose=False):
    """_build/logf_table.o: the glibc logf exception table, regenerated when its generator changes."""
    os.makedirs(BUILD, exist_ok=True)
    gen_src = os.path.join(CSRC, "gen_logf_table.c")
    deps = [gen_src, os.path.join(CSRC, "twlog.h")]
    table = os.path.join(BUILD, "logf_table.bin")
    obj = os.path.join(BUILD, "logf_table.o")
    env = dict(os.environ)
    env.pop("CXX", None)
    if not os.path.exists(table) or any(os.path.getmtime(d) > os.path.getmtime(table) for d in deps):
        gen = os.path.join(BUILD, "gen_logf_table")
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fopenmp", "-I", CSRC, "-o", gen, gen_src, "-lm"],
                       check=True, env=env)
        r = subprocess.run([gen, table], check=True, capture_output=True, text=True)
        if verbose:
            print("logf table:", r.stdout.strip(), "entries")
    asm = os.path.join(CSRC, "logf_table.S")
    if not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(table), os.path.getmtime(asm)):
        subprocess.run(["gcc", "-c", "-fPIC", "-Wa,-I," + BUILD, "-o", obj, asm], check=True, env=env)
    return obj


def _objects_stale(src, obj):
    """An object is rebuilt when its source or any header of csrc/ (or the C ABI header) is newer."""
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    heads = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    heads.append(os.path.join(os.path.dirname(HERE), "include", "twixtor_b200.h"))
    return os.path.getmtime(src) > t or any(os.path.getmtime(h) > t for h in heads)


def build(force=False, verbose=False):
    """Compiles every translation unit to an object in _build/ (in parallel), then links the library."""
    if not force and not stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    table_obj = logf_table_object(verbose)
    env = dict(os.environ)
    env.pop("CXX", None)  # host compiler: the system g++ (ccbin default)
    compile_flags = [f for f in FLAGS if f not in ("-shared", "-cudart", "shared")]
    # the fast mode's build of the solver's translation units: FMA contraction, approximate division
    # and square root, denormals flushed; its kernels in namespace tw::fast (TW_FAST_VARIANT)
    fast_flags = [{"-fmad=false": "-fmad=true", "-prec-div=true": "-prec-div=false",
                   "-prec-sqrt=true": "-prec-sqrt=false", "-ftz=false": "-ftz=true"}.get(f, f)
                  for f in compile_flags] + ["-DTW_FAST_VARIANT"]

    def compile_one(unit):
        name, fast = unit
        src = os.path.join(CSRC, name)
        obj = os.path.join(BUILD, name[:-3] + ("_fast.o" if fast else ".o"))
        if force or _objects_stale(src, obj):
            cmd = [NVCC] + (fast_flags if fast else compile_flags) + ["-c", "-o", obj, src]
            if verbose:
                print(" ".join(cmd))
            r = subprocess.run(cmd, env=env, cwd=CSRC, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {name}:\n{r.stdout}{r.stderr}")
        return obj

    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as pool:
        objs = list(pool.map(compile_one, [(n, False) for n in SOURCES] + [(n, True) for n in FAST_SOURCES]))
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "shared", "-o", LIB] + objs + [table_obj]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, env=env, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
