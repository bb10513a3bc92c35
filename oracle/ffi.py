"""ctypes bindings for the oracle libraries (test infrastructure only).

Restatement: oracle/_build/liboracle.so (oracle/cufe_oracle.c).
Reference:   oracle/_ref/<variant>/libref.so (cuFE's own CPU sources, see ref/build_ref.py).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")

Q = (16760833, 2147352577, 2130706433)


def _load(path):
    if not os.path.exists(path):
        raise FileNotFoundError(path + " (run python oracle/build.py)")
    return C.CDLL(path)


class Oracle:
    """The C restatement with runtime (n, l)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            L = _load(os.path.join(HERE, "_build", "liboracle.so"))
            L.or_params_new.restype = C.c_void_p
            L.or_params_new.argtypes = [C.c_int, C.c_int]
            L.or_params_free.argtypes = [C.c_void_p]
            L.or_params_export.argtypes = [C.c_void_p] + [C.c_void_p] * 7
            L.or_mod_prime.restype = C.c_uint32
            L.or_mod_prime.argtypes = [C.c_uint64, C.c_int]
            L.or_ct_forward.argtypes = [C.c_void_p, _u32p, C.c_int]
            L.or_gs_reverse.argtypes = [C.c_void_p, _u32p, C.c_int]
            L.or_ntt_generic.argtypes = [_u32p, C.c_int, C.c_uint32, _u32p, C.c_int, C.c_uint32]
            L.or_aes256_expand.argtypes = [_u8p, _u8p]
            L.or_aes256_block.argtypes = [_u8p, _u8p, _u8p]
            L.or_ctr_new.restype = C.c_void_p
            L.or_ctr_new.argtypes = [C.c_void_p, C.c_uint16]
            L.or_ctr_free.argtypes = [C.c_void_p]
            L.or_ctr_squeeze.argtypes = [C.c_void_p, _u8p, C.c_uint]
            L.or_ctr_counter.restype = C.c_uint32
            L.or_ctr_counter.argtypes = [C.c_void_p]
            L.or_gauss_call.argtypes = [C.c_void_p, C.c_void_p, C.c_int, _u32p, C.c_int]
            L.or_candidates.argtypes = [C.c_int, C.c_int, _u8p, _u64p, _u64p]
            L.or_modeB_refill.argtypes = [_u8p, C.c_uint32, _u8p]
            L.or_gauss_modeB_poly.argtypes = [C.c_void_p, _u8p, C.c_int, C.c_int, _u32p]
            L.or_sample_polya.argtypes = [C.c_void_p, _u8p, _u32p]
            L.or_setup.argtypes = [C.c_void_p, _u8p, C.c_void_p, _u8p, _u32p, _u32p]
            L.or_encrypt.argtypes = [C.c_void_p, _u32p, _u32p, _u8p, C.c_void_p, _u32p]
            L.or_keygen.argtypes = [C.c_void_p, _u32p, _u32p, _u32p]
            L.or_decrypt.argtypes = [C.c_void_p, _u32p, _u32p, _u32p, _u32p]
            L.or_decode.argtypes = [C.c_void_p, _u32p, _u32p, C.c_int]
            L.or_setup_modeB.argtypes = [C.c_void_p, _u8p, _u8p, _u32p, _u32p]
            L.or_encrypt_modeB.argtypes = [C.c_void_p, _u32p, _u32p, _u8p, C.c_int, _u32p]
            cls._lib = L
        return cls._lib

    def __init__(self, n, l):
        self.n, self.l = n, l
        self.L = self.lib()
        self.P = self.L.or_params_new(n, l)
        if not self.P:
            raise ValueError("bad (n, l)")

    def __del__(self):
        try:
            self.L.or_params_free(self.P)
        except Exception:
            pass

    # tables
    def tables(self):
        n = self.n
        psi = np.zeros(3 * n, np.uint32)
        psi_inv = np.zeros(3 * n, np.uint32)
        ninv = np.zeros(3, np.uint32)
        dm = np.zeros(3, np.uint32)
        p = np.zeros(1, np.uint32)
        ql = np.zeros(3, np.uint32)
        dl = np.zeros(3, np.uint32)
        self.L.or_params_export(self.P, psi.ctypes.data, psi_inv.ctypes.data, ninv.ctypes.data,
                                dm.ctypes.data, p.ctypes.data, ql.ctypes.data, dl.ctypes.data)
        q = int(ql[0]) | (int(ql[1]) << 32) | (int(ql[2]) << 64)
        delta = int(dl[0]) | (int(dl[1]) << 32) | (int(dl[2]) << 64)
        return dict(psi=psi.reshape(3, n), psi_inv=psi_inv.reshape(3, n), ninv=ninv,
                    delta_mod=dm, p=int(p[0]), q=q, delta=delta)

    # primitives
    def ntt(self, a, sel, inverse=False):
        a = np.ascontiguousarray(a, np.uint32).copy()
        (self.L.or_gs_reverse if inverse else self.L.or_ct_forward)(self.P, a, sel)
        return a

    def gauss(self, sig, key, ncalls):
        c = self.L.or_ctr_new(None if key is None else np.ascontiguousarray(key, np.uint8).ctypes.data, 0)
        out = np.zeros((ncalls, 3, self.n), np.uint32)
        buf = np.zeros(3 * self.n, np.uint32)
        for i in range(ncalls):
            self.L.or_gauss_call(self.P, c, sig, buf, self.n)
            out[i] = buf.reshape(3, self.n)
        ctr = self.L.or_ctr_counter(c)
        self.L.or_ctr_free(c)
        return out, ctr

    def gauss_modeB(self, rk, sig, poly):
        out = np.zeros(3 * self.n, np.uint32)
        self.L.or_gauss_modeB_poly(self.P, np.ascontiguousarray(rk, np.uint8), sig, poly, out)
        return out.reshape(3, self.n)

    def sample_polya(self, seed):
        a = np.zeros(3 * self.n, np.uint32)
        self.L.or_sample_polya(self.P, np.ascontiguousarray(seed, np.uint8), a)
        return a.reshape(3, self.n)

    # scheme
    def setup(self, seed_a, seed_s, seed_e):
        n, l = self.n, self.l
        mpk = np.zeros((l + 1) * 3 * n, np.uint32)
        msk = np.zeros(l * 3 * n, np.uint32)
        ss = None if seed_s is None else np.ascontiguousarray(seed_s, np.uint8)
        self.L.or_setup(self.P, np.ascontiguousarray(seed_a, np.uint8),
                        None if ss is None else ss.ctypes.data,
                        np.ascontiguousarray(seed_e, np.uint8), mpk, msk)
        return mpk.reshape(l + 1, 3, n), msk.reshape(l, 3, n)

    def encrypt(self, x, mpk, seed2, seed3=None):
        n, l = self.n, self.l
        ct = np.zeros((l + 1) * 3 * n, np.uint32)
        s3 = None if seed3 is None else np.ascontiguousarray(seed3, np.uint8)
        self.L.or_encrypt(self.P, np.ascontiguousarray(x, np.uint32), np.ascontiguousarray(mpk, np.uint32).ravel(),
                          np.ascontiguousarray(seed2, np.uint8), None if s3 is None else s3.ctypes.data, ct)
        return ct.reshape(l + 1, 3, n)

    def keygen(self, y, msk):
        sky = np.zeros(3 * self.n, np.uint32)
        self.L.or_keygen(self.P, np.ascontiguousarray(y, np.uint32),
                         np.ascontiguousarray(msk, np.uint32).ravel(), sky)
        return sky.reshape(3, self.n)

    def decrypt(self, ct, y, sky):
        dy = np.zeros(3 * self.n, np.uint32)
        self.L.or_decrypt(self.P, np.ascontiguousarray(ct, np.uint32).ravel(), np.ascontiguousarray(y, np.uint32),
                          np.ascontiguousarray(sky, np.uint32).ravel(), dy)
        return dy.reshape(3, self.n)

    def decode(self, dy, ncoeff=None):
        ncoeff = self.n if ncoeff is None else ncoeff
        out = np.zeros(ncoeff, np.uint32)
        self.L.or_decode(self.P, np.ascontiguousarray(dy, np.uint32).ravel(), out, ncoeff)
        return out

    def setup_modeB(self, a_coeff, seed2, seed3):
        n, l = self.n, self.l
        mpk = np.zeros((l + 1) * 3 * n, np.uint32)
        mpk[l * 3 * n:] = np.ascontiguousarray(a_coeff, np.uint32).ravel()
        msk = np.zeros(l * 3 * n, np.uint32)
        self.L.or_setup_modeB(self.P, np.ascontiguousarray(seed2, np.uint8),
                              np.ascontiguousarray(seed3, np.uint8), mpk, msk)
        return mpk.reshape(l + 1, 3, n), msk.reshape(l, 3, n)

    def encrypt_modeB(self, x, mpk, seed2):
        n, l = self.n, self.l
        x = np.ascontiguousarray(x, np.uint32).reshape(-1, l)
        rep = x.shape[0]
        ct = np.zeros(rep * (l + 1) * 3 * n, np.uint32)
        self.L.or_encrypt_modeB(self.P, x.ravel(), np.ascontiguousarray(mpk, np.uint32).ravel(),
                                np.ascontiguousarray(seed2, np.uint8), rep, ct)
        return ct.reshape(rep, l + 1, 3, n)


def aes256_expand(key):
    rk = np.zeros(240, np.uint8)
    Oracle.lib().or_aes256_expand(np.ascontiguousarray(key, np.uint8), rk)
    return rk


def aes256_block(rk, block):
    out = np.zeros(16, np.uint8)
    Oracle.lib().or_aes256_block(np.ascontiguousarray(rk, np.uint8), np.ascontiguousarray(block, np.uint8), out)
    return out


def ctr_stream(key, nblocks128, nonce=0):
    L = Oracle.lib()
    c = L.or_ctr_new(None if key is None else np.ascontiguousarray(key, np.uint8).ctypes.data, nonce)
    out = np.zeros(128 * nblocks128, np.uint8)
    L.or_ctr_squeeze(c, out, nblocks128)
    L.or_ctr_free(c)
    return out


def modeB_refill(rk, counter):
    out = np.zeros(384, np.uint8)
    Oracle.lib().or_modeB_refill(np.ascontiguousarray(rk, np.uint8), counter, out)
    return out


def candidates(sig, mapping, r):
    z = np.zeros(8, np.uint64)
    b = np.zeros(8, np.uint64)
    Oracle.lib().or_candidates(sig, mapping, np.ascontiguousarray(r, np.uint8), z, b)
    return z, b


class Reference:
    """The reference's own CPU sources (compiled dims fixed per variant)."""

    def __init__(self, variant="default"):
        path = os.path.join(HERE, "_ref", variant, "libref.so")
        L = _load(path)
        L.ref_n.restype = C.c_int
        L.ref_l.restype = C.c_int
        L.ref_queue_seeds.argtypes = [_u8p, C.c_int]
        L.ref_setup.argtypes = [_u32p, _u32p]
        L.ref_encrypt.argtypes = [_u32p, _u32p, _u32p]
        L.ref_keygen.argtypes = [_u32p, _u32p, _u32p]
        L.ref_decrypt.argtypes = [_u32p, _u32p, _u32p, _u32p, _u32p]
        L.ref_decode.argtypes = [_u32p, _u32p]
        L.ref_ct_forward.argtypes = [_u32p, C.c_int]
        L.ref_gs_reverse.argtypes = [_u32p, C.c_int]
        L.ref_sample_polya.argtypes = [_u8p, _u32p]
        L.ref_gauss.argtypes = [C.c_int, C.c_void_p, C.c_int, _u32p]
        L.ref_ctr_stream.argtypes = [C.c_void_p, C.c_int, _u8p]
        self.L = L
        self.n, self.l = L.ref_n(), L.ref_l()

    def _seeds(self, *seeds):
        s = np.concatenate([np.ascontiguousarray(x, np.uint8).ravel() for x in seeds])
        self.L.ref_queue_seeds(s, len(seeds))

    def setup(self, seed_a, seed_e):
        n, l = self.n, self.l
        self._seeds(seed_a, seed_e)
        mpk = np.zeros((l + 1) * 3 * n, np.uint32)
        msk = np.zeros(l * 3 * n, np.uint32)
        self.L.ref_setup(mpk, msk)
        return mpk.reshape(l + 1, 3, n), msk.reshape(l, 3, n)

    def encrypt(self, x, mpk, seed2):
        n, l = self.n, self.l
        self._seeds(seed2)
        ct = np.zeros((l + 1) * 3 * n, np.uint32)
        self.L.ref_encrypt(np.ascontiguousarray(x, np.uint32), np.ascontiguousarray(mpk, np.uint32).ravel().copy(), ct)
        return ct.reshape(l + 1, 3, n)

    def keygen(self, y, msk):
        sky = np.zeros(3 * self.n, np.uint32)
        self.L.ref_keygen(np.ascontiguousarray(y, np.uint32), np.ascontiguousarray(msk, np.uint32).ravel(), sky)
        return sky.reshape(3, self.n)

    def decrypt(self, ct, y, sky):
        dy = np.zeros(3 * self.n, np.uint32)
        dec = np.zeros(self.n, np.uint32)
        self.L.ref_decrypt(np.ascontiguousarray(ct, np.uint32).ravel().copy(), np.ascontiguousarray(y, np.uint32),
                           np.ascontiguousarray(sky, np.uint32).ravel().copy(), dy, dec)
        return dy.reshape(3, self.n), dec

    def decode(self, res):
        dec = np.zeros(self.n, np.uint32)
        self.L.ref_decode(np.ascontiguousarray(res, np.uint32).ravel(), dec)
        return dec

    def ntt(self, a, sel, inverse=False):
        a = np.ascontiguousarray(a, np.uint32).copy()
        (self.L.ref_gs_reverse if inverse else self.L.ref_ct_forward)(a, sel)
        return a

    def sample_polya(self, seed):
        a = np.zeros(3 * self.n, np.uint32)
        self.L.ref_sample_polya(np.ascontiguousarray(seed, np.uint8), a)
        return a.reshape(3, self.n)

    def gauss(self, sig, key, ncalls):
        out = np.zeros(ncalls * 3 * self.n, np.uint32)
        k = None if key is None else np.ascontiguousarray(key, np.uint8)
        self.L.ref_gauss(sig, None if k is None else k.ctypes.data, ncalls, out)
        return out.reshape(ncalls, 3, self.n)

    def ctr_stream(self, key, nblocks128):
        out = np.zeros(128 * nblocks128, np.uint8)
        k = None if key is None else np.ascontiguousarray(key, np.uint8)
        self.L.ref_ctr_stream(None if k is None else k.ctypes.data, nblocks128, out)
        return out


def canon(a, axis_moduli=-2):
    """canonical residues: the reference's mod_prime may return q_j in place of 0"""
    a = np.asarray(a, np.uint64)
    q = np.array(Q, np.uint64)
    shape = [1] * a.ndim
    shape[axis_moduli] = 3
    return (a % q.reshape(shape)).astype(np.uint32)


class ReferenceModeB:
    """The reference's GPU sampler kernels (src/sample_gpu.cu, src/AES.cuh, src/sampler.cuh) run
    on the host by oracle/ref/modeb/modeb_host.cpp: one block = one polynomial at n = 4096."""

    def __init__(self):
        L = _load(os.path.join(HERE, "_ref", "modeb", "libmodeb.so"))
        L.modeb_block.argtypes = [C.c_int, _u8p, C.c_int, _u32p]
        L.modeb_prepare_key.argtypes = [_u8p, _u8p]
        L.modeb_n.restype = C.c_int
        self.L = L
        self.n = L.modeb_n()

    def prepare_key(self, seed):
        rk = np.zeros(240, np.uint8)
        self.L.modeb_prepare_key(np.ascontiguousarray(seed, np.uint8), rk)
        return rk

    def poly(self, sig, seed, bid):
        out = np.zeros(3 * self.n, np.uint32)
        rc = self.L.modeb_block(sig, np.ascontiguousarray(seed, np.uint8), bid, out)
        if rc:
            raise RuntimeError("modeb_block failed: %d" % rc)
        return out.reshape(3, self.n)


class ReferenceCallers:
    """The reference's own callers of the GPU entry points (main.c, src/rlwe_sife.c, svm.cpp;
    n = 2048, l = 124) linked against cufe_b200/libcufe_b200.so: oracle/_ref/callers/."""

    PATH = os.path.join(HERE, "_ref", "callers", "libcallers.so")

    def __init__(self):
        L = _load(self.PATH)
        vp = C.c_void_p
        L.cl_n.restype = C.c_int
        L.cl_l.restype = C.c_int
        L.cl_queue_seeds.argtypes = [_u8p, C.c_int]
        L.cl_load_model.restype = vp
        L.cl_load_model.argtypes = [C.c_char_p]
        L.cl_free_model.argtypes = [vp]
        L.cl_model_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.cl_model_arrays.argtypes = [vp, vp, vp, vp, vp, vp]
        L.cl_predict_plain.restype = C.c_double
        L.cl_predict_plain.argtypes = [vp, _u32p]
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        for f in (L.cl_predict_cpu, L.cl_predict_gpu):
            f.restype = C.c_double
            f.argtypes = [vp, _u32p, _u32p, f64p, f64p]
        L.cl_setup.argtypes = [_u32p, _u32p]
        L.cl_encrypt.argtypes = [_u32p, _u32p, _u32p]
        L.cl_setup_gui.argtypes = [_u32p, _u32p]
        L.cl_encrypt_gui.argtypes = [_u32p, _u32p, _u32p, C.c_int]
        self.L = L
        self.n, self.l = L.cl_n(), L.cl_l()

    def seeds(self, *seeds):
        s = np.concatenate([np.ascontiguousarray(x, np.uint8).ravel() for x in seeds])
        self.L.cl_queue_seeds(s, len(s) // 32)

    def load_model(self, path):
        m = self.L.cl_load_model(path.encode())
        if not m:
            raise FileNotFoundError(path)
        k, t = C.c_int(0), C.c_int(0)
        self.L.cl_model_info(m, C.byref(k), C.byref(t))
        k, t = k.value, t.value
        arrays = {"label": np.zeros(k, np.int32), "nsv": np.zeros(k, np.int32),
                  "rho": np.zeros(k * (k - 1) // 2), "coef": np.zeros((k - 1, t)),
                  "sv": np.zeros((t, self.l), np.uint32)}
        self.L.cl_model_arrays(m, *(arrays[a].ctypes.data for a in ("label", "nsv", "rho", "coef", "sv")))
        return m, arrays

    def setup(self, seed_a, seed_e):
        mpk = np.zeros((self.l + 1, 3, self.n), np.uint32)
        msk = np.zeros((self.l, 3, self.n), np.uint32)
        self.seeds(seed_a, seed_e)
        self.L.cl_setup(mpk, msk)
        return mpk, msk

    def encrypt(self, x, mpk, seed2):
        c = np.zeros((self.l + 1, 3, self.n), np.uint32)
        self.seeds(seed2)
        self.L.cl_encrypt(np.ascontiguousarray(x, np.uint32), np.ascontiguousarray(mpk, np.uint32).copy(), c)
        return c

    def predict(self, model, c, msk, pairs, total_sv, gpu=False):
        """(label, dec[pairs], kvalue[total_sv]) of svm_predict_cpu (gpu: svm_predict_gpu)"""
        dec = np.zeros(pairs)
        kvalue = np.zeros(total_sv)
        f = self.L.cl_predict_gpu if gpu else self.L.cl_predict_cpu
        label = f(model, np.ascontiguousarray(c, np.uint32), np.ascontiguousarray(msk, np.uint32), dec, kvalue)
        return label, dec, kvalue
