"""Build the oracle libraries (test infrastructure only).

  oracle/_build/liboracle.so  -- the C restatement (oracle/cufe_oracle.c)
  oracle/_ref/<variant>/libref.so -- the reference's own CPU sources, when present here
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build_restatement(force=False):
    out = os.path.join(HERE, "_build")
    lib = os.path.join(out, "liboracle.so")
    src = os.path.join(HERE, "cufe_oracle.c")
    if os.path.exists(lib) and not force and os.path.getmtime(lib) >= os.path.getmtime(src):
        return lib
    os.makedirs(out, exist_ok=True)
    # -ffp-contract=off: the only fused multiply-adds are the explicit fma() calls
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-o", lib, src, "-lm"],
                   check=True)
    return lib


def build_all(force=False):
    build_restatement(force)
    sys.path.insert(0, os.path.join(HERE, "ref"))
    import build_ref  # noqa: E402
    build_ref.build_all(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("oracle built")
