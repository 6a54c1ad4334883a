"""Device-side helpers: uploads, the CSR pattern handle, CSR export, material tables."""

import ctypes

import numpy as np

from . import _lib


def torch():
    import torch as _t

    return _t


def device():
    _lib.require_cuda()
    t = torch()
    return t.device("cuda", t.cuda.current_device())


def upload(a, dtype):
    """numpy-like -> contiguous 1-D device tensor of ``dtype`` (np.float64 / np.int32 / np.uint8 / np.float32)."""
    t = torch()
    arr = np.ascontiguousarray(np.asarray(a, dtype=dtype).reshape(-1))
    if not arr.flags.writeable:
        arr = arr.copy()
    return t.from_numpy(arr).to(device(), non_blocking=False)


def to_host(x):
    """numpy copy of a device vector (synchronous read-back)."""
    return x.cpu().numpy()


def zeros(n, dtype="f64"):
    t = torch()
    dt = {"f64": t.float64, "f32": t.float32, "i32": t.int32}[dtype]
    return t.zeros(int(max(n, 1)), dtype=dt, device=device())


class _CudaArray:
    """Zero-copy view of device memory owned by the native library (``__cuda_array_interface__``)."""

    def __init__(self, ptr, n, typestr, owner):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2, "strides": None}
        self._owner = owner


class Pattern:
    """Owner of an ``snp_pattern`` (CSR pattern + element slot map) built on the device."""

    def __init__(self, elem_dofs, n_elems, dpe, n_rows, stream=None, handle=None, owned=True):
        self.n_rows = int(n_rows)
        self.dpe = int(dpe)
        self._owned = owned
        if handle is None:
            h = ctypes.c_void_p()
            _lib.call("snp_pattern_create", _lib.ptr(elem_dofs), int(n_elems), int(dpe), int(n_rows),
                      _lib.stream_ptr(stream), ctypes.byref(h))
            handle = h
        self.handle = handle
        nr, nnz, ne, d = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
        _lib.call("snp_pattern_info", self.handle, ctypes.byref(nr), ctypes.byref(nnz), ctypes.byref(ne), ctypes.byref(d))
        self.nnz = int(nnz.value)
        self.n_elems = int(ne.value)
        rp, ci, sl = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        _lib.call("snp_pattern_arrays", self.handle, ctypes.byref(rp), ctypes.byref(ci), ctypes.byref(sl))
        dg = ctypes.c_void_p()
        _lib.call("snp_pattern_diag", self.handle, ctypes.byref(dg))
        t = torch()
        dev = device()
        self.row_ptr = t.as_tensor(_CudaArray(rp.value, self.n_rows + 1, "<i4", self), device=dev)
        self.col_idx = t.as_tensor(_CudaArray(ci.value, max(self.nnz, 1), "<i4", self), device=dev)[: self.nnz]
        self.diag_pos = t.as_tensor(_CudaArray(dg.value, self.n_rows, "<i4", self), device=dev)
        sup = ctypes.c_int32()
        _lib.call("snp_curlcurl_rows_supported", self.handle, ctypes.byref(sup))
        self.rows_supported = bool(sup.value)

    def to_scipy(self, values, drop_zeros=False):
        """Host scipy ``csr_array`` with this pattern and the given device values."""
        from scipy.sparse import csr_array

        t = torch()
        t.cuda.synchronize()
        data = values[: self.nnz].double().cpu().numpy()
        A = csr_array((data, self.col_idx.cpu().numpy().astype(np.int32), self.row_ptr.cpu().numpy().astype(np.int32)),
                      shape=(self.n_rows, self.n_rows))
        A.has_sorted_indices = True
        if drop_zeros:
            A.eliminate_zeros()
        return A

    def to_torch(self, values):
        """Device ``torch.sparse_csr_tensor`` (float64 values, int32 indices) with this pattern and
        the given device values; every structural entry is kept, exact zeros included.  The
        index arrays are copies, so the tensor outlives the pattern."""
        import warnings

        t = torch()
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", UserWarning)  # torch's notes on sparse CSR being in beta
            return t.sparse_csr_tensor(self.row_ptr.clone(), self.col_idx.clone(), values[: self.nnz],
                                       size=(self.n_rows, self.n_rows))

    def __del__(self):
        try:
            if self._owned and self.handle is not None and _lib._lib is not None:
                _lib.load().snp_pattern_destroy(self.handle)
        except Exception:
            pass
        self.handle = None


def reluctance_tables(reluctance):
    """(n_int, rel_c, rel_x) device tensors as the Cython layer marshals a reluctance
    (``fem_c/interface_c.pyx:226-234``); unknown types print the reference's message and
    fall back to the constant-zero table, as it does."""
    spl_x = np.zeros((0,))
    spl_c = np.zeros((1,))
    ts = reluctance.get_type_spec()
    if ts == 1:
        spl_c, spl_x = reluctance.get_spline_information()
    elif ts == 0:
        spl_c = np.array([float(reluctance.value)])
    else:
        print("Type specifyer of reluctance not found!")
    n_int = len(spl_x) - 1
    c = upload(np.asarray(spl_c).flatten(), np.float64)
    x = upload(spl_x if len(spl_x) else np.zeros(1), np.float64)
    return n_int, c, x


def permeability_tables(permeability):
    """(type, degree, n_ctrl, knots, ctrl, H_min, mu_H_min) as ``fem_c/interface_c.pyx:56-68``."""
    spl_t, spl_c, spl_k, H_min, mu_H_min, n = np.zeros((1,)), np.zeros((1,)), 1, 0.0, 4 * np.pi * 1e-7, 0
    ts = permeability.get_type_spec()
    if ts == 0:
        mu_H_min = float(np.asarray(permeability.evaluate_mu(0.0)).reshape(-1)[0])
    elif ts == 1:
        spl_t, spl_c, spl_k, H_min, mu_H_min = permeability.get_spline_information()
        n = len(spl_t) - spl_k - 1
    else:
        print("Type specifyer of permeability not found!")
    return (int(ts) if ts in (0, 1) else 0, int(spl_k), int(n), upload(spl_t, np.float64), upload(spl_c, np.float64),
            float(H_min), float(mu_H_min))


def check_affine(curls, d_phi, n_quad):
    """Raise unless the tables are the same at every quadrature point (first-order tetrahedra)."""
    d = np.asarray(d_phi, dtype=np.float64).reshape(n_quad, -1)
    c = np.asarray(curls, dtype=np.float64).reshape(-1, n_quad, 18)
    if not (np.array_equal(d, np.broadcast_to(d[:1], d.shape)) and np.array_equal(c, np.broadcast_to(c[:, :1], c.shape))):
        raise ValueError("d_phi/curls vary across quadrature points: only first-order (affine) tetrahedra are supported")
