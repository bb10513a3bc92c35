"""Build the reference's own CPU path (cuFE src/*.c, compiled unmodified from where the
sources lie in the reference tree given by --root or $CUFE_REFERENCE_ROOT) into
oracle/_ref/<variant>/libref.so, and the reference's GPU sampler kernels as host code into
oracle/_ref/modeb/libmodeb.so.

TEST INFRASTRUCTURE ONLY: the resulting libraries are the pinned oracle that the C
restatement (oracle/cufe_oracle.c) and the golden fixtures are checked against, and the
CPU baseline timed by bench.py --impl reference.

Recipe (no copying of reference sources; outputs only under oracle/_ref/):
  * the reference headers are used as shipped for the `default` variant (n=4096, l=785);
    other (n, l) variants pre-include a generated params/consts header (-include) whose
    include guards (PARAMS_H, CONSTS_H) turn the shipped params.h/consts.h into no-ops;
  * <gmp.h> is the declaration shim in oracle/ref/shim, linked to the system libgmp.so.10;
  * src/randombytes.c is replaced by oracle/ref/ref_glue.c (queued seeds) at link time;
  * -ftrivial-auto-var-init=zero makes the never-initialised AES contexts of
    rlwe_sife_setup/encrypt deterministic (all-zero round keys, counter 0);
  * -O3 with AVX2/FMA/AES-NI (the reference Makefile uses -march=native -mavx2; the
    explicit x86-64-v3 target keeps the library runnable on any AVX2 host and keeps
    the FMA contraction of the Bernoulli polynomial that -march=native gives).
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT = os.path.join(ORACLE, "_ref")
UNITS = ["aes256ctr.c", "arith_rns.c", "crt.c", "gauss.c", "ntt.c", "rlwe_sife.c", "sample.c"]
CFLAGS = ["-O3", "-fomit-frame-pointer", "-march=x86-64-v3", "-maes", "-fPIC", "-w",
          "-ftrivial-auto-var-init=zero"]

Q = [16760833, 2147352577, 2130706433]
PSI8192 = [3689, 1689795, 456478]
VARIANTS = {  # name -> (n, l); None = shipped headers
    "default": None,
    "n4096_l784": (4096, 784),
    "n2048_l124": (2048, 124),
    "n1024_l16": (1024, 16),
    "n256_l8": (256, 8),
}


def _bitrev(x, bits):
    return int(format(x, "0%db" % bits)[::-1], 2) if bits else 0


def _root(j, n):
    q = Q[j]
    if 2 * n <= 8192:
        return pow(PSI8192[j], 8192 // (2 * n), q)
    raise ValueError("variants above n=4096 are not built")


def gen_headers(n, l, d):
    qfull = Q[0] * Q[1] * Q[2]
    p = 64 * l + 1
    delta = qfull // p
    c1 = pow(Q[0], -1, Q[1])
    c2 = pow(Q[0] * Q[1], -1, Q[2])
    with open(os.path.join(d, "gen_params.h"), "w") as f:
        f.write("/* generated by oracle/ref/build_ref.py: n=%d l=%d */\n" % (n, l))
        f.write("#ifndef PARAMS_H\n#define PARAMS_H\n#include <stdint.h>\n#include <stdlib.h>\n")
        f.write("#define Malloc(type,n) (type *)malloc((n)*sizeof(type))\n")
        f.write("#define max_data 1\n#define CLOCKS_PER_MS 2700000\n#define PERF\n#define CPU\n#define GPU\n")
        f.write('static const char SIFE_Q_str[] = "%d";\n' % qfull)
        f.write("#define SIFE_LOGQ_BYTE 88\n#define SIFE_NMODULI 3\n")
        f.write("static const uint64_t SIFE_CRT_CONSTS[SIFE_NMODULI]={0, %d, %d};\n" % (c1, c2))
        f.write("static const uint32_t SIFE_MOD_Q_I[SIFE_NMODULI] = {%d, %d, %d};\n" % tuple(Q))
        f.write("#define SIFE_B_x 4\n#define SIFE_B_y 16\n#define SIFE_L %d\n#define SIFE_N %d\n" % (l, n))
        f.write("#define SIFE_SIGMA 1\n")
        f.write('static const char SIFE_P_str[] = "%d";\n' % p)
        f.write('static const char SIFE_SCALE_M_str[]="%d";\n' % delta)
        f.write("static const uint64_t SIFE_SCALE_M_MOD_Q_I[SIFE_NMODULI]={%d, %d, %d};\n"
                % tuple(delta % q for q in Q))
        f.write("#endif\n")
    logn = n.bit_length() - 1
    with open(os.path.join(d, "gen_consts.h"), "w") as f:
        f.write("/* generated by oracle/ref/build_ref.py: n=%d */\n" % n)
        f.write("#ifndef CONSTS_H\n#define CONSTS_H\n#include <stdint.h>\n")
        f.write("static const uint32_t SIFE_NTT_NINV[SIFE_NMODULI]={%s};\n"
                % ", ".join(str(pow(n, -1, q)) for q in Q))
        for name, sign in (("psi", 1), ("psi_inv", -1)):
            rows = []
            for j, q in enumerate(Q):
                w = pow(_root(j, n), sign, q)
                rows.append("{" + ", ".join(str(pow(w, _bitrev(k, logn), q)) for k in range(n)) + "}")
            f.write("uint32_t %s[SIFE_NMODULI][SIFE_N] = {%s};\n" % (name, ",\n".join(rows)))
        f.write("#endif\n")


def ref_root(root=None):
    """the reference tree: the argument, else $CUFE_REFERENCE_ROOT; there is no default"""
    root = root or os.environ.get("CUFE_REFERENCE_ROOT")
    if not root:
        raise RuntimeError("reference tree not given: pass root= / --root or set CUFE_REFERENCE_ROOT")
    return root


def build_variant(root, name, dims, force=False):
    d = os.path.join(OUT, name)
    lib = os.path.join(d, "libref.so")
    if os.path.exists(lib) and not force:
        return lib
    os.makedirs(d, exist_ok=True)
    pre = []
    if dims is not None:
        gen_headers(dims[0], dims[1], d)
        pre = ["-include", os.path.join(d, "gen_params.h")]
    src_dir = os.path.join(root, "src")
    inc = ["-I", src_dir, "-I", os.path.join(HERE, "shim")]
    objs = []
    for unit in UNITS + ["GLUE"]:
        src = os.path.join(HERE, "ref_glue.c") if unit == "GLUE" else os.path.join(src_dir, unit)
        obj = os.path.join(d, os.path.basename(src) + ".o")
        extra = list(pre)
        if dims is not None and unit == "ntt.c":
            extra += ["-include", os.path.join(d, "gen_consts.h")]
        cmd = ["gcc", "-c", src, "-o", obj] + CFLAGS + extra + inc
        subprocess.run(cmd, check=True)
        objs.append(obj)
    subprocess.run(["gcc", "-shared", "-o", lib] + objs + ["-l:libgmp.so.10", "-lm"], check=True)
    return lib


# --------------------------------------------------------------- GPU counter mapping (mode B)
MODEB_FUNCS = ["__global__ void gaussian_sampler_S1_gpu(", "__global__ void gaussian_sampler_S2_gpu(",
               "__device__ uint32_t add_mod_ntt_gpu_2(", "__global__ void gaussian_sampler_S3_gpu("]
MODEB_FLAGS = ["-O2", "-fPIC", "-shared", "-std=c++17", "-w", "-fwrapv", "-fno-strict-aliasing",
               "-ffp-contract=fast", "-march=x86-64-v3", "-ftrivial-auto-var-init=zero"]


def extract_functions(text, heads):
    """the text of each function definition starting with one of `heads`, unmodified, in file
    order (from its head to the matching closing brace)"""
    out = []
    for head in heads:
        i = text.index(head)
        j = text.index("{", i)
        depth = 0
        for k in range(j, len(text)):
            if text[k] == "{":
                depth += 1
            elif text[k] == "}":
                depth -= 1
                if depth == 0:
                    out.append((i, text[i:k + 1]))
                    break
        else:
            raise ValueError("unbalanced braces after " + head)
    return [t for _, t in sorted(out)]


def build_modeb(root, force=False):
    """oracle/_ref/modeb/libmodeb.so: the reference's GPU sampler kernels (src/sample_gpu.cu) and
    device headers compiled as host C++ by oracle/ref/modeb/modeb_host.cpp"""
    d = os.path.join(OUT, "modeb")
    lib = os.path.join(d, "libmodeb.so")
    shim = os.path.join(HERE, "modeb")
    newest = max(os.path.getmtime(os.path.join(shim, f)) for f in os.listdir(shim))
    if os.path.exists(lib) and not force and os.path.getmtime(lib) >= newest:
        return lib
    os.makedirs(d, exist_ok=True)
    src_dir = os.path.join(root, "src")
    with open(os.path.join(src_dir, "sample_gpu.cu")) as f:
        text = f.read()
    with open(os.path.join(d, "sample_gpu_kernels.inc"), "w") as f:
        f.write("/* extracted from the reference's src/sample_gpu.cu by oracle/ref/build_ref.py; "
                "not committed */\n")
        for body in extract_functions(text, MODEB_FUNCS):
            f.write(body + "\n\n")
    cmd = (["g++"] + MODEB_FLAGS + ["-I", shim, "-I", src_dir, "-I", d, "-o", lib,
                                    os.path.join(shim, "modeb_host.cpp")])
    subprocess.run(cmd, check=True)
    return lib


# --------------------------------------------------------------- the reference's own callers
CALLERS_VARIANT = ("n2048_l124", (2048, 124))


def build_callers(root, force=False):
    """oracle/_ref/callers/libcallers.so: the reference's callers of the GPU entry points
    (main.c with main renamed, src/*.c including rlwe_sife.c's *_gui wrappers, svm/svm.cpp)
    compiled unmodified at n = 2048, l = 124 and linked against cufe_b200/libcufe_b200.so,
    which must resolve rlwe_sife_{setup,encrypt,keygen}_gpu and rlwe_sife_decrypt_gmp_gpu
    (the link fails otherwise).  Requires the library to be built first."""
    name, dims = CALLERS_VARIANT
    d = os.path.join(OUT, "callers")
    lib = os.path.join(d, "libcallers.so")
    cufe_dir = os.path.join(os.path.dirname(ORACLE), "cufe_b200")
    cufe_lib = os.path.join(cufe_dir, "libcufe_b200.so")
    if not os.path.exists(cufe_lib):
        raise FileNotFoundError(cufe_lib + " (build the library first)")
    if os.path.exists(lib) and not force and os.path.getmtime(lib) >= os.path.getmtime(cufe_lib):
        return lib
    os.makedirs(d, exist_ok=True)
    gen_headers(dims[0], dims[1], d)
    src_dir = os.path.join(root, "src")
    pre = ["-include", os.path.join(d, "gen_params.h")]
    inc = ["-I", src_dir, "-I", root, "-I", os.path.join(HERE, "shim")]
    objs = []
    units = [os.path.join(src_dir, u) for u in UNITS]
    units += [os.path.join(root, "main.c"), os.path.join(HERE, "callers_glue.c")]
    for src in units:
        obj = os.path.join(d, os.path.basename(src) + ".o")
        extra = list(pre)
        if src.endswith("ntt.c"):
            extra += ["-include", os.path.join(d, "gen_consts.h")]
        if src.endswith("main.c"):
            extra += ["-Dmain=ref_main"]
        subprocess.run(["gcc", "-c", src, "-o", obj] + CFLAGS + extra + inc, check=True)
        objs.append(obj)
    svm_obj = os.path.join(d, "svm.o")
    subprocess.run(["g++", "-c", os.path.join(root, "svm", "svm.cpp"), "-o", svm_obj, "-O3", "-fPIC", "-w"],
                   check=True)
    objs.append(svm_obj)
    link = (["g++", "-shared", "-o", lib] + objs +
            ["-L", cufe_dir, "-l:libcufe_b200.so", "-Wl,-rpath,$ORIGIN/../../../cufe_b200",
             "-Wl,--wrap=malloc", "-Wl,--wrap=free", "-Wl,--no-undefined", "-l:libgmp.so.10", "-lm"])
    subprocess.run(link, check=True)
    return lib


def build_all(root=None, force=False):
    root = ref_root(root)
    if not os.path.isdir(os.path.join(root, "src")):
        return False
    for name, dims in VARIANTS.items():
        build_variant(root, name, dims, force)
    build_modeb(root, force)
    build_callers(root, force)
    return True


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--root", help="the reference tree (default: $CUFE_REFERENCE_ROOT)")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    ok = build_all(a.root, force=a.force)
    print("built" if ok else "reference sources absent; nothing built")
