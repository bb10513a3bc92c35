"""The reference's own callers link against this library (CPU only, no device touched).

oracle/ref/build_ref.py compiles the reference's main.c and src/*.c (src/rlwe_sife.c holds the
*_gui wrappers that call the GPU entry points, main.c the svm_predict_gpu prediction) unmodified
and links them with --no-undefined against cufe_b200/libcufe_b200.so.  Here: the result loads,
its four GPU entry points are undefined in it (declared extern at src/rlwe_sife.c:23-29 and
main.c:22-28) and resolve to the definitions this library exports.
"""
import ctypes as C
import os
import subprocess

import pytest

from oracle.ffi import ReferenceCallers

DROPIN = ("rlwe_sife_setup_gpu", "rlwe_sife_encrypt_gpu", "rlwe_sife_keygen_gpu", "rlwe_sife_decrypt_gmp_gpu")


@pytest.mark.skipif(not os.path.exists(ReferenceCallers.PATH), reason="reference callers not built")
def test_reference_callers_bind_to_the_dropin_symbols():
    import cufe_b200 as cf
    und = subprocess.run(["nm", "-D", "--undefined-only", ReferenceCallers.PATH], capture_output=True,
                         text=True, check=True).stdout.split()
    for name in DROPIN:
        assert name in und, name
    needed = subprocess.run(["readelf", "-d", ReferenceCallers.PATH], capture_output=True, text=True,
                            check=True).stdout
    assert "libcufe_b200.so" in needed
    R = ReferenceCallers()
    assert (R.n, R.l) == (2048, 124)
    mine = cf.lib()
    for name in DROPIN:
        theirs = C.cast(getattr(R.L, name), C.c_void_p).value
        assert theirs == C.cast(getattr(mine, name), C.c_void_p).value, name
