"""Calls MEX gateways built against the in-repo MEX stand-in (emclarity_b200/mex/shim): ours in
emclarity_b200/mex/_shim/ and the reference's own MEX sources compiled into oracle/_ref/.

Arguments: numpy arrays / Python scalars become host mxArrays, torch CUDA tensors become
gpuArrays (MATLAB dims are the reverse of the torch shape).  Returned gpuArrays are copied
into torch CUDA tensors, host arrays into numpy arrays."""
import ctypes as C
import glob
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLASS = {np.dtype(np.float64): 6, np.dtype(np.float32): 7, np.dtype(np.bool_): 3, np.dtype(np.int8): 8,
         np.dtype(np.uint8): 9, np.dtype(np.int16): 10, np.dtype(np.uint16): 11, np.dtype(np.int32): 12,
         np.dtype(np.uint32): 13, np.dtype(np.int64): 14, np.dtype(np.uint64): 15}
NP_OF = {v: k for k, v in CLASS.items()}
SIZE_T = C.c_size_t

_cudart = None


def cudart():
    global _cudart
    if _cudart is None:
        import torch  # noqa: F401  (loads the CUDA runtime torch uses)
        for name in ("libcudart.so.12", "libcudart.so"):
            try:
                _cudart = C.CDLL(name)
                break
            except OSError:
                continue
        if _cudart is None:
            cands = glob.glob("/usr/local/cuda/lib64/libcudart.so*")
            _cudart = C.CDLL(cands[0])
        _cudart.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    return _cudart


class MexLib:
    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        L.emc_shim_wrap_host.restype = C.c_void_p
        L.emc_shim_wrap_host.argtypes = [C.c_void_p, SIZE_T, C.POINTER(SIZE_T), C.c_int, C.c_int]
        L.emc_shim_wrap_gpu.restype = C.c_void_p
        L.emc_shim_wrap_gpu.argtypes = [C.c_void_p, SIZE_T, C.POINTER(SIZE_T), C.c_int, C.c_int]
        L.emc_shim_call.restype = C.c_int
        L.emc_shim_call.argtypes = [C.c_int, C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]
        L.emc_shim_last_error.restype = C.c_char_p
        L.mxGetData.restype = C.c_void_p
        L.mxGetData.argtypes = [C.c_void_p]
        L.mxGetClassID.restype = C.c_int
        L.mxGetClassID.argtypes = [C.c_void_p]
        L.mxIsComplex.restype = C.c_bool
        L.mxIsComplex.argtypes = [C.c_void_p]
        L.emc_shim_is_gpu.restype = C.c_bool
        L.emc_shim_is_gpu.argtypes = [C.c_void_p]
        L.emc_shim_dims.restype = C.POINTER(SIZE_T)
        L.emc_shim_dims.argtypes = [C.c_void_p, C.POINTER(SIZE_T)]
        L.mxDestroyArray.argtypes = [C.c_void_p]

    def _wrap(self, x, keep):
        import torch
        if isinstance(x, torch.Tensor):
            cplx = 1 if x.is_complex() else 0
            base = torch.float32 if x.dtype == torch.complex64 else x.dtype
            np_dt = {torch.float32: np.float32, torch.float64: np.float64, torch.int32: np.int32}[base]
            dims = (SIZE_T * max(1, x.dim()))(*reversed(list(x.shape)))
            keep.append(x)
            return self.lib.emc_shim_wrap_gpu(C.c_void_p(x.data_ptr()), max(1, x.dim()), dims,
                                              CLASS[np.dtype(np_dt)], cplx)
        a = np.asarray(x)
        cplx = 0
        if np.iscomplexobj(a):
            cplx = 1
            a = np.ascontiguousarray(a.astype(np.complex64 if a.dtype == np.complex64 else np.complex128))
            base = np.dtype(np.float32 if a.dtype == np.complex64 else np.float64)
        else:
            base = a.dtype
        a = np.ascontiguousarray(a.T) if a.ndim > 1 else np.ascontiguousarray(a.reshape(-1))
        keep.append(a)
        shape = list(np.asarray(x).shape) if np.asarray(x).ndim else [1]
        if len(shape) == 1:
            shape = [shape[0], 1]
        dims = (SIZE_T * len(shape))(*shape)
        return self.lib.emc_shim_wrap_host(a.ctypes.data_as(C.c_void_p), len(shape), dims, CLASS[base], cplx)

    def _unwrap(self, p):
        import torch
        L = self.lib
        nd = SIZE_T(0)
        dp = L.emc_shim_dims(p, C.byref(nd))
        dims = [dp[i] for i in range(nd.value)]
        cls = L.mxGetClassID(p)
        cplx = L.mxIsComplex(p)
        dt = NP_OF[cls]
        if L.emc_shim_is_gpu(p):
            tdt = {np.dtype(np.float32): torch.complex64 if cplx else torch.float32,
                   np.dtype(np.float64): torch.complex128 if cplx else torch.float64}[dt]
            shape = list(reversed(dims))
            while len(shape) > 1 and shape[0] == 1 and len(shape) > 3:
                shape = shape[1:]
            t = torch.empty(shape, dtype=tdt, device="cuda")
            nbytes = t.numel() * t.element_size()
            torch.cuda.synchronize()
            assert cudart().cudaMemcpy(C.c_void_p(t.data_ptr()), C.c_void_p(L.mxGetData(p)), nbytes, 4) == 0
            return t
        n = int(np.prod(dims))
        buf = (C.c_char * (n * np.dtype(dt).itemsize * (2 if cplx else 1))).from_address(L.mxGetData(p))
        a = np.frombuffer(bytes(buf), dtype=dt)
        if cplx:
            a = a.view(np.complex64 if dt == np.float32 else np.complex128)
        return a.reshape(list(reversed(dims))).T.copy() if len(dims) > 1 else a.copy()

    def __call__(self, nlhs, *args):
        keep = []
        prhs = (C.c_void_p * max(1, len(args)))(*[self._wrap(a, keep) for a in args])
        plhs = (C.c_void_p * max(1, nlhs))()
        rc = self.lib.emc_shim_call(nlhs, plhs, len(args), prhs)
        for p in prhs:
            self.lib.mxDestroyArray(p)
        if rc != 0:
            raise RuntimeError(self.lib.emc_shim_last_error().decode())
        outs = []
        for i in range(nlhs):
            if plhs[i]:
                outs.append(self._unwrap(plhs[i]))
                self.lib.mxDestroyArray(plhs[i])
            else:
                outs.append(None)
        return outs


def ours(name):
    return MexLib(os.path.join(ROOT, "emclarity_b200", "mex", "_shim", "lib%s.so" % name))


def reference(name):
    return MexLib(os.path.join(ROOT, "oracle", "_ref", "libref_%s.so" % name))


def have_reference():
    return all(os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_%s.so" % n))
               for n in ("mexXform3d", "mexCTF", "mexFFT"))
