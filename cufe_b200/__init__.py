"""cufe_b200: B200-native (sm_100a) RLWE inner-product functional encryption.

Python binding over the C ABI of libcufe_b200.so (include/cufe_b200.h).  Device buffers are
torch CUDA tensors (plumbing only); every computation runs in the library's own kernels.
There is no CPU fallback: importing works without a GPU, but every compute call needs the
shared library and a CUDA device and raises otherwise.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcufe_b200.so")

OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of device memory",
          -4: "sampler status set", -5: "no CUDA device"}
SIGMA1, SIGMA2, SIGMA3 = 0, 1, 2
OBJ_MPK, OBJ_MSK, OBJ_CT, OBJ_SKY, OBJ_DY = 1, 2, 3, 4, 5
NTT_VARIANTS = 9  # CUFE_NTT_VARIANTS
Q = (16760833, 2147352577, 2130706433)

_lib = None


class CufeError(RuntimeError):
    def __init__(self, code, what):
        self.code = code
        msg = _lib.cufe_last_error().decode() if _lib is not None else ""
        super().__init__("%s: %s (%d) %s" % (what, ERRORS.get(code, "error"), code, msg))


def compile_library(force=False):
    """Compile the CUDA sources into the in-tree shared library (cufe_b200/build.py)."""
    import importlib
    return importlib.import_module("cufe_b200.build").build(force=force)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libcufe_b200.so is not built (python -m cufe_b200.build)")
        L = C.CDLL(LIB_PATH)
        vp, i, ll = C.c_void_p, C.c_int, C.c_longlong
        L.cufe_last_error.restype = C.c_char_p
        L.cufe_version.restype = C.c_char_p
        sig = {
            "cufe_create": [C.POINTER(vp), i, i, i],
            "cufe_destroy": [vp],
            "cufe_sync": [vp, vp],
            "cufe_ctx_stream": [vp],
            "cufe_params": [vp, vp, vp],
            "cufe_profile_enable": [vp, i],
            "cufe_profile_read": [vp, i, vp, vp, vp],
            "cufe_profile_reset": [vp],
            "cufe_profile_launches": [vp],
            "cufe_tables": [vp, vp, vp],
            "cufe_setup": [vp, vp, vp, vp, vp, vp, vp],
            "cufe_setup_gpu_map": [vp, vp, vp, vp, vp, vp],
            "cufe_encrypt": [vp, i, vp, vp, vp, vp, vp, vp],
            "cufe_encrypt_gpu_map": [vp, i, vp, vp, vp, vp, vp],
            "cufe_keygen": [vp, i, vp, i, vp, vp, vp],
            "cufe_decrypt": [vp, i, vp, i, vp, i, vp, vp, vp],
            "cufe_decrypt_noalloc": [vp, vp, i, vp, i, vp, vp, vp],
            "cufe_decode": [vp, i, vp, i, vp, vp],
            "cufe_tune_encrypt": [vp, i, vp, vp, vp, vp, vp, vp, vp, vp],
            "cufe_tune_decrypt_coef0": [vp, i, vp, i, vp, i, vp, vp, vp, vp, vp],
            "cufe_decrypt_coef0_form": [vp, i, i, vp, i, vp, i, vp, vp, vp, vp],
            "cufe_svm_tune": [vp, i, vp, vp, vp, vp],
            "cufe_batch_tune": [vp, i, vp, vp, vp, vp],
            "cufe_decrypt_coef0": [vp, i, vp, i, vp, i, vp, vp, vp, vp],
            "cufe_sample_cpu_map": [vp, i, i, vp, i, vp, vp],
            "cufe_sample_gpu_map": [vp, i, vp, i, i, vp, vp],
            "cufe_sample_polya": [vp, vp, vp, vp],
            "cufe_ring_create": [C.POINTER(vp), i, i, vp, i],
            "cufe_ring_destroy": [vp],
            "cufe_ring_info": [vp, vp, vp, vp, vp],
            "cufe_ntt_forward": [vp, vp, ll, vp],
            "cufe_ntt_inverse": [vp, vp, ll, vp],
            "cufe_ring_tune": [vp, ll, vp, vp],
            "cufe_batch_create": [C.POINTER(vp), i, vp, vp, C.c_size_t, i],
            "cufe_batch_destroy": [vp],
            "cufe_batch_setup": [vp, vp, vp, vp, vp],
            "cufe_batch_bind": [vp, vp, vp, vp, vp, vp, vp],
            "cufe_batch_run": [vp, vp],
            "cufe_batch_replay": [vp, vp],
            "cufe_batch_status": [vp],
            "cufe_batch_info": [vp, vp, vp, vp, vp],
            "cufe_batch_instance": [vp, i, vp, vp, vp, vp],
            "cufe_batch_profile": [vp, i],
            "cufe_batch_profile_read": [vp, vp, vp],
            "cufe_batch_graph_kernels": [vp],
            "cufe_batch_profile_groups": [vp, i, vp, vp, vp],
            "cufe_svm_create": [C.POINTER(vp), vp, i, i, vp, i, vp, vp, vp, vp, vp, vp],
            "cufe_svm_predict": [vp, i, vp, vp, vp, vp, vp],
            "cufe_svm_destroy": [vp],
            "cufe_server_create": [C.POINTER(vp), i, vp, vp, C.c_size_t, C.c_size_t, i],
            "cufe_server_destroy": [vp],
            "cufe_server_setup": [vp, vp, vp, vp],
            "cufe_server_encrypt": [vp, i, vp, vp, vp, C.c_double],
            "cufe_server_keygen": [vp, i, vp, C.c_double],
            "cufe_server_decrypt": [vp, ll, ll, C.c_double],
            "cufe_server_poll": [vp, i],
            "cufe_server_pending": [vp, vp, vp],
            "cufe_server_result": [vp, ll, vp, vp, vp, vp],
            "cufe_server_read": [vp, ll, vp, C.c_size_t],
            "cufe_server_release": [vp, ll],
            "cufe_server_stats": [vp, vp, vp, vp],
            "cufe_server_limits": [vp, i, C.c_double],
            "cufe_ring_set_variant": [vp, i, i],
            "cufe_ring_get_variant": [vp, vp, vp],
            "cufe_sampler_refills": [i, i, i],
            "cufe_sampler_call_search": [i],
            "cufe_serialized_bytes": [vp, i, i],
            "cufe_serialize": [vp, i, i, vp, vp, vp],
            "cufe_deserialize": [vp, i, i, vp, C.c_size_t, vp, vp],
            "cufe_dropin_configure": [i, i, i],
            "cufe_dropin_status": [],
            "rlwe_sife_setup_gpu": [vp, vp, vp, vp, vp],
            "rlwe_sife_encrypt_gpu": [vp, vp, vp, vp, vp, i, vp],
            "rlwe_sife_keygen_gpu": [vp, vp, vp, i, vp],
            "rlwe_sife_decrypt_gmp_gpu": [vp, vp, vp, vp, i, vp],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = None if name.startswith("rlwe_sife_") else C.c_int
        L.cufe_sampler_refills.restype = C.c_longlong
        L.cufe_serialized_bytes.restype = C.c_longlong
        L.cufe_profile_launches.restype = C.c_longlong
        for name in ("cufe_server_encrypt", "cufe_server_keygen", "cufe_server_decrypt"):
            getattr(L, name).restype = C.c_longlong
        L.cufe_server_shed.argtypes = [vp]
        L.cufe_server_shed.restype = C.c_longlong
        L.cufe_server_now.argtypes = []
        L.cufe_server_now.restype = C.c_double
        _lib = L
    return _lib


def _refills_s3(n, l):
    """refills per encryption stream of the sigma_3 sampler (CPU mapping)"""
    return int(lib().cufe_sampler_refills(SIGMA3, l, n))


def _check(rc, what):
    if rc != OK:
        raise CufeError(rc, what)


def _ptr(t):
    """device or host address of a torch tensor / numpy array (None -> NULL)"""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


def _seeds(s):
    if s is None:
        return None
    a = np.ascontiguousarray(np.asarray(s, dtype=np.uint8).reshape(-1))
    return a


def u32(t):
    """torch int32 tensor -> numpy uint32 copy on the host"""
    return t.detach().cpu().numpy().view(np.uint32)


def _stream(stream, device):
    """stream handle for a call: the given one, else torch's current stream on device"""
    if stream is not None:
        return stream
    import torch
    return torch.cuda.current_stream(device).cuda_stream or None


def _dev(shape, device):
    import torch
    return torch.empty(shape, dtype=torch.int32, device=device)


def to_dev(a, device="cuda"):
    """uint32 words on the device (int32 tensor of the same bits)"""
    import torch
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint32))
    return torch.from_numpy(a.view(np.int32)).to(device)


def bytes_to_dev(a, device="cuda"):
    """bytes (seeds) on the device, unchanged: a uint8 tensor"""
    import torch
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint8))
    return torch.from_numpy(a).to(device)


class Context:
    """An IPFE parameter set (ring degree n, vector length l) on one device."""

    def __init__(self, n, l, device=0):
        L = lib()
        self.n, self.l, self.device = n, l, device
        h = C.c_void_p()
        _check(L.cufe_create(C.byref(h), n, l, device), "cufe_create")
        self.h = h
        p = np.zeros(1, np.uint32)
        dm = np.zeros(3, np.uint32)
        _check(L.cufe_params(h, p.ctypes.data, dm.ctypes.data), "cufe_params")
        self.p, self.delta_mod = int(p[0]), dm
        self.dev = "cuda:%d" % device

    def close(self):
        if getattr(self, "h", None):
            lib().cufe_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return lib().cufe_ctx_stream(self.h)

    def sync(self, stream=None):
        _check(lib().cufe_sync(self.h, _stream(stream, self.device)), "cufe_sync")

    def profile(self, on=True):
        _check(lib().cufe_profile_enable(self.h, int(on)), "cufe_profile_enable")

    def profile_reset(self):
        _check(lib().cufe_profile_reset(self.h), "cufe_profile_reset")

    def profile_launches(self):
        """kernel launches of this context while profiling was on, since the last reset"""
        n = lib().cufe_profile_launches(self.h)
        if n < 0:
            raise CufeError(int(n), "cufe_profile_launches")
        return int(n)

    def profile_read(self):
        """{group name: (kernel launches, total ms)} since the last reset"""
        names = C.create_string_buffer(64 * 64)
        launches = np.zeros(64, np.int64)
        ms = np.zeros(64, np.float64)
        k = lib().cufe_profile_read(self.h, 64, names, launches.ctypes.data, ms.ctypes.data)
        if k < 0:
            raise CufeError(k, "cufe_profile_read")
        raw = names.raw
        return {raw[64 * i:64 * i + 64].split(b"\0")[0].decode(): (int(launches[i]), float(ms[i])) for i in range(k)}

    def tables(self):
        psi = np.zeros((3, self.n), np.uint32)
        ipsi = np.zeros((3, self.n), np.uint32)
        _check(lib().cufe_tables(self.h, psi.ctypes.data, ipsi.ctypes.data), "cufe_tables")
        return psi, ipsi

    # ---- buffers
    def mpk_buf(self):
        return _dev((self.l + 1, 3, self.n), self.dev)

    def msk_buf(self):
        return _dev((self.l, 3, self.n), self.dev)

    def ct_buf(self, batch):
        return _dev((batch, self.l + 1, 3, self.n), self.dev)

    # ---- scheme (device tensors; ordered on torch's current stream unless a stream is given)
    def setup(self, seed_a, seed_s, seed_e, mpk=None, msk=None, stream=None):
        mpk = self.mpk_buf() if mpk is None else mpk
        msk = self.msk_buf() if msk is None else msk
        sa, ss, se = _seeds(seed_a), _seeds(seed_s), _seeds(seed_e)
        _check(lib().cufe_setup(self.h, _ptr(sa), _ptr(ss), _ptr(se), _ptr(mpk), _ptr(msk), _stream(stream, self.device)), "cufe_setup")
        return mpk, msk

    def setup_gpu_map(self, a_coeff, seed2, seed3, mpk=None, msk=None, stream=None):
        import torch
        mpk = self.mpk_buf() if mpk is None else mpk
        msk = self.msk_buf() if msk is None else msk
        mpk[self.l].copy_(torch.as_tensor(a_coeff).to(mpk.device).reshape(3, self.n))
        s2, s3 = _seeds(seed2), _seeds(seed3)
        _check(lib().cufe_setup_gpu_map(self.h, _ptr(s2), _ptr(s3), _ptr(mpk), _ptr(msk),
                                         _stream(stream, self.device)), "cufe_setup_gpu_map")
        return mpk, msk

    def encrypt(self, x, mpk, seeds2, seeds3=None, ct=None, stream=None):
        batch = x.shape[0]
        ct = self.ct_buf(batch) if ct is None else ct
        s2, s3 = _seeds(seeds2), _seeds(seeds3)
        _check(lib().cufe_encrypt(self.h, batch, _ptr(x), _ptr(mpk), _ptr(s2), _ptr(s3), _ptr(ct), _stream(stream, self.device)),
               "cufe_encrypt")
        return ct

    def encrypt_gpu_map(self, x, mpk, seed2, ct=None, stream=None):
        batch = x.shape[0]
        ct = self.ct_buf(batch) if ct is None else ct
        s2 = _seeds(seed2)
        _check(lib().cufe_encrypt_gpu_map(self.h, batch, _ptr(x), _ptr(mpk), _ptr(s2), _ptr(ct), _stream(stream, self.device)),
               "cufe_encrypt_gpu_map")
        return ct

    def keygen(self, y, msk, y_signed=False, sky=None, stream=None):
        nkeys = y.shape[0]
        sky = _dev((nkeys, 3, self.n), self.dev) if sky is None else sky
        _check(lib().cufe_keygen(self.h, nkeys, _ptr(y), int(y_signed), _ptr(msk), _ptr(sky), _stream(stream, self.device)), "cufe_keygen")
        return sky

    def decrypt(self, ct, y, sky, y_signed=False, dy=None, stream=None):
        nct, nkeys = ct.shape[0], y.shape[0]
        dy = _dev((nct, nkeys, 3, self.n), self.dev) if dy is None else dy
        _check(lib().cufe_decrypt(self.h, nct, _ptr(ct), nkeys, _ptr(y), int(y_signed), _ptr(sky), _ptr(dy), _stream(stream, self.device)),
               "cufe_decrypt")
        return dy

    def decrypt_noalloc(self, ct, y, sky, y_signed=False, dy=None, stream=None):
        """Decryption of one ciphertext ct[1][l+1][3][n] with up to 4 keys; the library call
        allocates no device memory.  When dy is None this wrapper allocates the output with
        torch, so a caller on a fixed device-memory budget passes its own dy[1][nkeys][3][n]."""
        nkeys = y.shape[0]
        if ct.shape[0] != 1:
            raise ValueError("decrypt_noalloc takes exactly one ciphertext, got %d" % ct.shape[0])
        if dy is None:
            dy = _dev((1, nkeys, 3, self.n), self.dev)
        elif tuple(dy.shape) != (1, nkeys, 3, self.n):
            raise ValueError("dy must have shape (1, %d, 3, %d), got %s" % (nkeys, self.n, tuple(dy.shape)))
        _check(lib().cufe_decrypt_noalloc(self.h, _ptr(ct), nkeys, _ptr(y), int(y_signed), _ptr(sky), _ptr(dy),
                                          _stream(stream, self.device)), "cufe_decrypt_noalloc")
        return dy

    def tune_encrypt(self, x, mpk, seeds2, seeds3, ct=None, stream=None):
        """time one and two instances per thread group for this batch size on these inputs (the
        ciphertexts land in ct either way); the context keeps the faster.  -> (choice, [ms1, ms2])"""
        batch = x.shape[0]
        ct = self.ct_buf(batch) if ct is None else ct
        s2, s3 = _seeds(seeds2), _seeds(seeds3)
        ch, ms = C.c_int(0), (C.c_float * 2)()
        _check(lib().cufe_tune_encrypt(self.h, batch, _ptr(x), _ptr(mpk), _ptr(s2), _ptr(s3), _ptr(ct), C.byref(ch),
                                       ms, _stream(stream, self.device)), "cufe_tune_encrypt")
        return ch.value, list(ms)

    def tune_decrypt_coef0(self, ct, y, sky, y_signed=False, out=None, stream=None):
        """time the five coefficient-0 decrypt forms for (nct, nkeys); -> (form, ms[5])"""
        nct, nkeys = ct.shape[0], y.shape[0]
        out = _dev((nct, nkeys), self.dev) if out is None else out
        ch, ms = C.c_int(0), (C.c_float * 5)()
        _check(lib().cufe_tune_decrypt_coef0(self.h, nct, _ptr(ct), nkeys, _ptr(y), int(y_signed), _ptr(sky), _ptr(out),
                                             C.byref(ch), ms, _stream(stream, self.device)), "cufe_tune_decrypt_coef0")
        return ch.value, list(ms)

    def decrypt_coef0_form(self, form, ct, y, sky, y_signed=False, d0=None, out=None, stream=None):
        """decrypt_coef0 in a given form (0 per pair, 1..4 tile shapes)"""
        nct, nkeys = ct.shape[0], y.shape[0]
        out = _dev((nct, nkeys), self.dev) if out is None else out
        _check(lib().cufe_decrypt_coef0_form(self.h, form, nct, _ptr(ct), nkeys, _ptr(y), int(y_signed), _ptr(sky),
                                             _ptr(d0), _ptr(out), _stream(stream, self.device)),
               "cufe_decrypt_coef0_form")
        return out

    def decrypt_coef0(self, ct, y, sky, y_signed=False, d0=None, out=None, stream=None):
        """decrypt and decode coefficient 0 of every (ciphertext, key) pair: out[nct][nkeys]"""
        nct, nkeys = ct.shape[0], y.shape[0]
        out = _dev((nct, nkeys), self.dev) if out is None else out
        _check(lib().cufe_decrypt_coef0(self.h, nct, _ptr(ct), nkeys, _ptr(y), int(y_signed), _ptr(sky), _ptr(d0),
                                        _ptr(out), _stream(stream, self.device)), "cufe_decrypt_coef0")
        return out

    def decode(self, dy, ncoeff=None, out=None, stream=None):
        ncoeff = self.n if ncoeff is None else ncoeff
        count = dy.numel() // (3 * self.n)
        out = _dev((count, ncoeff), self.dev) if out is None else out
        _check(lib().cufe_decode(self.h, count, _ptr(dy), ncoeff, _ptr(out), _stream(stream, self.device)), "cufe_decode")
        return out

    # ---- serialization
    def serialize(self, kind, t, stream=None):
        """pack count objects of `kind` (OBJ_*) from device tensor t: a uint8 device tensor"""
        import torch
        count = t.numel() // (self._polys(kind) * self.n)
        nbytes = lib().cufe_serialized_bytes(self.h, kind, count)
        if nbytes < 0:
            raise CufeError(int(nbytes), "cufe_serialized_bytes")
        out = torch.empty(nbytes, dtype=torch.uint8, device=t.device)
        _check(lib().cufe_serialize(self.h, kind, count, _ptr(t), _ptr(out), _stream(stream, self.device)),
               "cufe_serialize")
        return out

    def _polys(self, kind):
        return {OBJ_MPK: (self.l + 1) * 3, OBJ_MSK: self.l * 3, OBJ_CT: (self.l + 1) * 3, OBJ_SKY: 3, OBJ_DY: 3}[kind]

    def deserialize(self, kind, buf, count, out=None, stream=None):
        import torch
        polys = self._polys(kind)
        out = torch.empty((count, polys // 3, 3, self.n), dtype=torch.int32, device=buf.device) if out is None else out
        _check(lib().cufe_deserialize(self.h, kind, count, _ptr(buf), buf.numel(), _ptr(out),
                                      _stream(stream, self.device)), "cufe_deserialize")
        return out

    # ---- samplers
    def sample_cpu_map(self, sig, keys, calls, nstreams=None, out=None, stream=None):
        k = _seeds(keys)
        ns = nstreams if nstreams is not None else (1 if k is None else len(k) // 32)
        out = _dev((ns, calls, 3, self.n), self.dev) if out is None else out
        _check(lib().cufe_sample_cpu_map(self.h, sig, ns, _ptr(k), calls, _ptr(out), _stream(stream, self.device)), "cufe_sample_cpu_map")
        return out

    def sample_gpu_map(self, sig, key, poly0, npolys, out=None, stream=None):
        out = _dev((npolys, 3, self.n), self.dev) if out is None else out
        k = _seeds(key)
        _check(lib().cufe_sample_gpu_map(self.h, sig, _ptr(k), poly0, npolys, _ptr(out), _stream(stream, self.device)),
               "cufe_sample_gpu_map")
        return out

    def sample_polya(self, seed, out=None, stream=None):
        out = _dev((3, self.n), self.dev) if out is None else out
        sd = _seeds(seed)
        _check(lib().cufe_sample_polya(self.h, _ptr(sd), _ptr(out), _stream(stream, self.device)), "cufe_sample_polya")
        return out


class Ring:
    """RNS ring for the negacyclic NTT kernels (k primes, degree n)."""

    def __init__(self, n, k, primes=None, device=0):
        L = lib()
        self.n, self.k, self.device = n, k, device
        h = C.c_void_p()
        pr = None if primes is None else np.ascontiguousarray(primes, np.uint32)
        _check(L.cufe_ring_create(C.byref(h), n, k, _ptr(pr), device), "cufe_ring_create")
        self.h = h
        self.primes = np.zeros(k, np.uint32)
        self.roots = np.zeros(k, np.uint32)
        self.psi = np.zeros((k, n), np.uint32)
        self.psi_inv = np.zeros((k, n), np.uint32)
        _check(L.cufe_ring_info(h, self.primes.ctypes.data, self.roots.ctypes.data, self.psi.ctypes.data,
                                self.psi_inv.ctypes.data), "cufe_ring_info")

    def close(self):
        if getattr(self, "h", None):
            lib().cufe_ring_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, data, stream=None):
        npoly = data.numel() // (self.k * self.n)
        _check(lib().cufe_ntt_forward(self.h, _ptr(data), npoly, _stream(stream, self.device)), "cufe_ntt_forward")
        return data

    def inverse(self, data, stream=None):
        npoly = data.numel() // (self.k * self.n)
        _check(lib().cufe_ntt_inverse(self.h, _ptr(data), npoly, _stream(stream, self.device)), "cufe_ntt_inverse")
        return data

    def tune(self, npoly, stream=None):
        """time the NTT_VARIANTS kernel variants in both directions on npoly scratch polynomials
        and keep the fastest; returns {"fwd": [ms v1..], "inv": [...], "variant": (fwd, inv)}"""
        ms = np.zeros(2 * NTT_VARIANTS, np.float32)
        _check(lib().cufe_ring_tune(self.h, npoly, ms.ctypes.data, _stream(stream, self.device)), "cufe_ring_tune")
        return {"fwd": [float(x) for x in ms[:NTT_VARIANTS]], "inv": [float(x) for x in ms[NTT_VARIANTS:]],
                "variant": self.variant}

    @property
    def variant(self):
        f, v = C.c_int(0), C.c_int(0)
        _check(lib().cufe_ring_get_variant(self.h, C.byref(f), C.byref(v)), "cufe_ring_get_variant")
        return f.value, v.value

    def set_variant(self, fwd, inv):
        _check(lib().cufe_ring_set_variant(self.h, fwd, inv), "cufe_ring_set_variant")


class Batch:
    """Many independent IPFE instances of different (n_i, l_i), each with its own master key
    pair, stepped together: encrypt x_i, keygen y_i (signed), decrypt and decode the
    inner product (coefficient 0 of d_y, in [0, p_i], p_i = 64 l_i + 1)."""

    def __init__(self, n, l, max_chunk_bytes=0, device=0):
        import torch
        self.n = np.ascontiguousarray(n, np.int32)
        self.l = np.ascontiguousarray(l, np.int32)
        assert self.n.shape == self.l.shape and self.n.ndim == 1
        self.count, self.device = len(self.n), device
        self.dev = torch.device("cuda", device)
        h = C.c_void_p()
        _check(lib().cufe_batch_create(C.byref(h), self.count, self.n.ctypes.data, self.l.ctypes.data,
                                       max_chunk_bytes, device), "cufe_batch_create")
        self.h = h
        self.x_off = np.zeros(self.count + 1, np.uint64)
        ch, kb, sb = C.c_int(0), C.c_size_t(0), C.c_size_t(0)
        _check(lib().cufe_batch_info(h, self.x_off.ctypes.data, C.byref(ch), C.byref(kb), C.byref(sb)),
               "cufe_batch_info")
        self.chunks, self.key_bytes, self.scratch_bytes = ch.value, kb.value, sb.value
        self._bound = None

    def close(self):
        if getattr(self, "h", None):
            lib().cufe_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setup(self, seeds_a, seeds_s, seeds_e, stream=None):
        a, s_, e = _seeds(seeds_a), _seeds(seeds_s), _seeds(seeds_e)
        _check(lib().cufe_batch_setup(self.h, _ptr(a), _ptr(s_), _ptr(e), _stream(stream, self.device)),
               "cufe_batch_setup")

    def pack(self, rows):
        """concatenate per-instance vectors (instance i of length l_i) in the batch's layout"""
        return np.concatenate([np.asarray(r).reshape(-1) for r in rows])

    def bind(self, x, y, seeds2, seeds3, out=None, d0=None):
        """device tensors: x uint32/int32 [sum l], y int32 [sum l], seeds [count][32] uint8"""
        import torch
        for t in (seeds2, seeds3):
            if t.dtype != torch.uint8 or t.numel() != 32 * self.count:
                raise ValueError("seeds must be uint8 device tensors of [count][32] bytes")
        out = torch.empty(self.count, dtype=torch.int32, device=self.dev) if out is None else out
        _check(lib().cufe_batch_bind(self.h, _ptr(x), _ptr(y), _ptr(seeds2), _ptr(seeds3), _ptr(out), _ptr(d0)),
               "cufe_batch_bind")
        self._bound = (x, y, seeds2, seeds3, out, d0)  # keep the buffers alive
        return out

    def run(self, stream=None):
        _check(lib().cufe_batch_run(self.h, _stream(stream, self.device)), "cufe_batch_run")

    def replay(self, stream=None):
        _check(lib().cufe_batch_replay(self.h, _stream(stream, self.device)), "cufe_batch_replay")

    def tune(self, budgets, stream=None):
        """re-chunk at each scratch budget (bytes), time an eager step, keep the fastest;
        -> (chosen budget, ms per budget, -1 where it did not fit)"""
        b = (C.c_size_t * len(budgets))(*budgets)
        ms = (C.c_float * len(budgets))()
        chosen = C.c_size_t(0)
        _check(lib().cufe_batch_tune(self.h, len(budgets), b, C.byref(chosen), ms, _stream(stream, self.device)),
               "cufe_batch_tune")
        ch, kb, sb = C.c_int(0), C.c_size_t(0), C.c_size_t(0)
        _check(lib().cufe_batch_info(self.h, None, C.byref(ch), C.byref(kb), C.byref(sb)), "cufe_batch_info")
        self.chunks, self.scratch_bytes = ch.value, sb.value
        return chosen.value, list(ms)

    def profile(self, on):
        """kernel timing of eager steps (run()); on clears the totals"""
        _check(lib().cufe_batch_profile(self.h, int(on)), "cufe_batch_profile")

    def profile_read(self):
        """(summed kernel milliseconds, kernels launched) of the profiled eager steps"""
        ms, k = C.c_double(0), C.c_longlong(0)
        _check(lib().cufe_batch_profile_read(self.h, C.byref(ms), C.byref(k)), "cufe_batch_profile_read")
        return ms.value, k.value

    def profile_groups(self):
        """{group name: (kernels launched, ms)} of the profiled eager steps"""
        names = C.create_string_buffer(64 * 64)
        launches = (C.c_longlong * 64)()
        ms = (C.c_double * 64)()
        k = lib().cufe_batch_profile_groups(self.h, 64, names, launches, ms)
        if k < 0:
            raise CufeError(k, "cufe_batch_profile_groups")
        return {names.raw[64 * i:64 * i + 64].split(b"\0")[0].decode(): (launches[i], ms[i]) for i in range(k)}

    def graph_kernels(self):
        r = lib().cufe_batch_graph_kernels(self.h)
        if r < 0:
            raise CufeError(r, "cufe_batch_graph_kernels")
        return r

    def status(self):
        _check(lib().cufe_batch_status(self.h), "cufe_batch_status")

    def instance(self, i):
        """(mpk, msk, sky, ct) device addresses of instance i (ct None unless available)"""
        ptrs = [C.c_void_p() for _ in range(4)]
        _check(lib().cufe_batch_instance(self.h, i, *[C.byref(p) for p in ptrs]), "cufe_batch_instance")
        return tuple(p.value for p in ptrs)

    def fetch(self, addr, words):
        """copy `words` uint32 from a device address of this batch into a numpy array"""
        import torch

        class _View:  # a device range exposed through __cuda_array_interface__ (no copy)
            __cuda_array_interface__ = {"shape": (words,), "typestr": "<i4", "data": (addr, False), "version": 2}

        t = torch.as_tensor(_View(), device=self.dev)
        torch.cuda.synchronize(self.dev)
        return t.cpu().numpy().view(np.uint32)


class Server:
    """Request server over resident tenants (continuous batching): submit encrypt / keygen /
    decrypt requests, poll() to make progress, read results by request id."""

    QUEUED, RUNNING, DONE, RELEASED, SHED = 0, 1, 2, 3, 4

    def __init__(self, n, l, arena_bytes=0, tick_bytes=0, device=0):
        self.n = np.ascontiguousarray(n, np.int32)
        self.l = np.ascontiguousarray(l, np.int32)
        self.device = device
        h = C.c_void_p()
        _check(lib().cufe_server_create(C.byref(h), len(self.n), self.n.ctypes.data, self.l.ctypes.data,
                                        arena_bytes, tick_bytes, device), "cufe_server_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().cufe_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def now():
        return lib().cufe_server_now()

    def setup(self, seeds_a, seeds_s, seeds_e):
        a, s_, e = _seeds(seeds_a), _seeds(seeds_s), _seeds(seeds_e)
        _check(lib().cufe_server_setup(self.h, _ptr(a), _ptr(s_), _ptr(e)), "cufe_server_setup")

    def _id(self, r, what):
        if r < 0:
            raise CufeError(int(r), what)
        return int(r)

    def encrypt(self, tenant, x, seed2, seed3, t_arrival=-1.0):
        x = np.ascontiguousarray(x, np.uint32)
        s2, s3 = _seeds(seed2), _seeds(seed3)
        return self._id(lib().cufe_server_encrypt(self.h, tenant, x.ctypes.data, s2.ctypes.data, s3.ctypes.data,
                                                  t_arrival), "cufe_server_encrypt")

    def keygen(self, tenant, y, t_arrival=-1.0):
        y = np.ascontiguousarray(y, np.int32)
        return self._id(lib().cufe_server_keygen(self.h, tenant, y.ctypes.data, t_arrival), "cufe_server_keygen")

    def decrypt(self, ct, sk, t_arrival=-1.0):
        return self._id(lib().cufe_server_decrypt(self.h, ct, sk, t_arrival), "cufe_server_decrypt")

    def poll(self, wait=False):
        r = lib().cufe_server_poll(self.h, int(wait))
        if r < 0:
            raise CufeError(r, "cufe_server_poll")
        return r

    def pending(self):
        q, t = C.c_longlong(0), C.c_int(0)
        _check(lib().cufe_server_pending(self.h, C.byref(q), C.byref(t)), "cufe_server_pending")
        return q.value, t.value

    def drain(self):
        while True:
            q, t = self.pending()
            if q == 0 and t == 0:
                return
            self.poll(wait=t > 0)

    def result(self, rid):
        st, v, ta, td = C.c_int(0), C.c_uint32(0), C.c_double(0), C.c_double(0)
        _check(lib().cufe_server_result(self.h, rid, C.byref(st), C.byref(v), C.byref(ta), C.byref(td)),
               "cufe_server_result")
        return st.value, v.value, ta.value, td.value

    def read(self, rid, words):
        out = np.zeros(words, np.uint32)
        _check(lib().cufe_server_read(self.h, rid, out.ctypes.data, words), "cufe_server_read")
        return out

    def release(self, rid):
        _check(lib().cufe_server_release(self.h, rid), "cufe_server_release")

    def stats(self):
        t, d, f = C.c_longlong(0), C.c_longlong(0), C.c_size_t(0)
        _check(lib().cufe_server_stats(self.h, C.byref(t), C.byref(d), C.byref(f)), "cufe_server_stats")
        shed = lib().cufe_server_shed(self.h)
        if shed < 0:
            raise CufeError(int(shed), "cufe_server_shed")
        return {"ticks": t.value, "done": d.value, "ct_free_bytes": f.value, "shed": int(shed)}

    def limits(self, max_tick_requests=0, max_queue_s=0.0):
        """Overload control: at most max_tick_requests per tick (0: memory limits only); requests
        queued longer than max_queue_s when a tick is formed are shed (0: never)."""
        _check(lib().cufe_server_limits(self.h, int(max_tick_requests), float(max_queue_s)),
               "cufe_server_limits")


class SvmModel:
    """An encrypted linear-SVM predictor on a Context: the support vectors' function keys are
    derived once; predict() decrypts every (ciphertext, support vector) inner product and takes
    the libsvm one-against-one vote on the device."""

    def __init__(self, ctx, sv, nsv, sv_coef, rho, label, msk, signed=True, stream=None):
        self.ctx = ctx
        sv = np.ascontiguousarray(sv, np.int32)
        assert sv.ndim == 2 and sv.shape[1] == ctx.l
        self.lsv = sv.shape[0]
        self.nr_class = len(nsv)
        self.npairs = self.nr_class * (self.nr_class - 1) // 2
        nsv = np.ascontiguousarray(nsv, np.int32)
        coef = np.ascontiguousarray(sv_coef, np.float64).reshape(self.nr_class - 1, self.lsv)
        rho = np.ascontiguousarray(rho, np.float64).reshape(self.npairs)
        label = np.ascontiguousarray(label, np.int32)
        h = C.c_void_p()
        _check(lib().cufe_svm_create(C.byref(h), ctx.h, self.nr_class, self.lsv, sv.ctypes.data, int(signed),
                                     nsv.ctypes.data, coef.ctypes.data, rho.ctypes.data, label.ctypes.data, _ptr(msk),
                                     _stream(stream, ctx.device)), "cufe_svm_create")
        self.h = h

    def predict(self, ct, labels=None, kvalue=None, dec=None, stream=None):
        import torch
        nct = ct.shape[0]
        labels = torch.empty(nct, dtype=torch.int32, device=ct.device) if labels is None else labels
        _check(lib().cufe_svm_predict(self.h, nct, _ptr(ct), _ptr(labels), _ptr(kvalue), _ptr(dec),
                                      _stream(stream, self.ctx.device)), "cufe_svm_predict")
        return labels

    def tune(self, ct, stream=None):
        """pick the coefficient-0 decrypt form for this many test vectors; -> (form, ms[5])"""
        ch, ms = C.c_int(0), (C.c_float * 5)()
        _check(lib().cufe_svm_tune(self.h, ct.shape[0], _ptr(ct), C.byref(ch), ms, _stream(stream, self.ctx.device)),
               "cufe_svm_tune")
        return ch.value, list(ms)

    def close(self):
        if getattr(self, "h", None):
            lib().cufe_svm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
