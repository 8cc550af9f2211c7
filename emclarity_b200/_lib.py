"""ctypes binding of libemc_b200.so (the C-ABI declared in include/emc_b200.h).

The shared library is built in-tree by ``emclarity_b200.build``.  Loading fails loudly
when it is missing: there is no CPU fallback for any entry point.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libemc_b200.so")

EMC_OK = 0
EMC_E_ARG = -1
EMC_E_CUDA = -2
EMC_E_OOM = -3
EMC_E_TIMEOUT = -4
EMC_E_UNSUPPORTED = -5

INTERP_LINEAR = 0
INTERP_CUBIC = 1
INTERP_LINEAR_BORDER = 2
DTYPE_F32 = 0
DTYPE_BF16 = 1


class EmcError(RuntimeError):
    def __init__(self, status, where, detail):
        super().__init__("%s failed: status %d (%s): %s" % (where, status, _status_name(status), detail))
        self.status = status


def _status_name(s):
    return {0: "ok", -1: "EMC_E_ARG", -2: "EMC_E_CUDA", -3: "EMC_E_OOM", -4: "EMC_E_TIMEOUT",
            -5: "EMC_E_UNSUPPORTED"}.get(s, "unknown")


class ParticleDesc(C.Structure):
    _fields_ = [("spectrum", C.c_void_p), ("energy", C.c_double), ("prior", C.c_double * 9),
                ("shift", C.c_float * 3), ("box", C.c_int), ("ref_id", C.c_int),
                ("orient_begin", C.c_int), ("orient_count", C.c_int), ("wedge", C.c_void_p)]


class SearchHit(C.Structure):
    _fields_ = [("cc", C.c_float), ("orient", C.c_int), ("peak", C.c_int * 3)]


class CtfParams(C.Structure):
    _fields_ = [("pixel_size", C.c_float), ("wavelength", C.c_float), ("cs_mm", C.c_float),
                ("amp_contrast", C.c_float), ("defocus1", C.c_float), ("defocus2", C.c_float),
                ("astig_deg", C.c_float)]


class MrcHeader(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("mode", C.c_int),
                ("mx", C.c_int), ("my", C.c_int), ("mz", C.c_int), ("cell", C.c_float * 3),
                ("pixel_size", C.c_float * 3), ("dmin", C.c_float), ("dmax", C.c_float), ("dmean", C.c_float),
                ("rms", C.c_float), ("origin", C.c_float * 3), ("ext_bytes", C.c_int), ("imod_stamp", C.c_int),
                ("imod_flags", C.c_int), ("data_offset", C.c_long), ("byte_swapped", C.c_int)]


_vp, _i, _d, _f = C.c_void_p, C.c_int, C.c_double, C.c_float
_pd, _pi, _pf = C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_float)

# name -> (restype, argtypes)
SIGNATURES = {
    "emc_status_string": (C.c_char_p, [_i]),
    "emc_last_error": (C.c_char_p, []),
    "emc_version": (C.c_char_p, []),
    "emc_define_matrix": (_i, [_pd, _i, _pd]),
    "emc_euler_search": (_i, [C.c_char_p, _d, _d, _d, _d, _pd, _pi]),
    "emc_xform3d_create": (_i, [_vp, _i, _i, _i, _i, C.POINTER(_vp), _vp]),
    "emc_xform3d_apply": (_i, [_vp, _pd, _i, _pf, _i, _i, _vp, _vp]),
    "emc_xform3d_destroy": (_i, [_vp]),
    "emc_fft_plan": (_i, [_i, _pi, _i, C.POINTER(_vp)]),
    "emc_fft_r2c": (_i, [_vp, _vp, _vp, _vp]),
    "emc_fft_c2r": (_i, [_vp, _vp, _vp, _vp]),
    "emc_fft_destroy": (_i, [_vp]),
    "emc_ctf2d": (_i, [C.POINTER(CtfParams), _i, _i, _i, _i, _i, _vp, _vp]),
    "emc_binary_wedge": (_i, [_i, _f, _f, _i, _i, _vp, _vp]),
    "emc_centred_to_half": (_i, [_vp, _i, _i, _i, _i, _vp, _vp]),
    "emc_mask_sphere": (_i, [_pi, _pd, _pd, _d, _vp, _vp]),
    "emc_cref_filter": (_i, [_pd, _pd, _i, _pd, _pd, _i, _d, _pi, _f, _vp, _vp]),
    "emc_ctf2d_exposure": (_i, [C.POINTER(CtfParams), _i, _i, _i, _i, _i, _f, _f, _vp, _vp]),
    "emc_sf3d": (_i, [_i, _i, C.POINTER(C.c_uint), _pf, _pf, _pf, _pf, _pf, _pf, _pf, C.c_uint, _pf, _pf, _pf,
                      _vp, _vp]),
    "emc_wedge_ctf_weight": (_i, [_i, _f, _f, C.POINTER(CtfParams), _i, _vp, _vp]),
    "emc_pad3d": (_i, [_vp, _i, _i, _i, _pi, _pi, _f, _i, _vp, _vp]),
    "emc_bandpass3d": (_i, [_i, _i, _i, _f, _f, _f, _f, _vp, _vp]),
    "emc_band_limit_center_normalize": (_i, [_vp, _i, _i, _i, _pi, _pi, _i, _vp, _vp, _vp]),
    "emc_xcf_rotational": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, _pd, _vp]),
    "emc_xcf_translational": (_i, [_vp, _vp, _i, _i, _i, _vp, _i, _pd, _pd, _vp, _vp]),
    "emc_particle_spectrum": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "emc_particle_spectra": (_i, [_i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "emc_particle_template": (_i, [_i, _vp, _vp, _vp]),
    "emc_search_create": (_i, [C.POINTER(_vp)]),
    "emc_search_add_reference": (_i, [_vp, _vp, _i, _vp, _vp, _i, _pi, _vp]),
    "emc_search_set_orientations": (_i, [_vp, _pd, _i]),
    "emc_search_configure": (_i, [_vp, _i, _i, _i]),
    "emc_search_run": (_i, [_vp, C.POINTER(ParticleDesc), _i, _vp, _vp, _vp, _vp]),
    "emc_search_run_energies": (_i, [_vp, C.POINTER(ParticleDesc), _i, _vp, _vp, _vp, _vp, _vp]),
    "emc_search_run_host": (_i, [_vp, C.POINTER(ParticleDesc), _i, _pf, _pi, C.POINTER(SearchHit), _vp]),
    "emc_search_destroy": (_i, [_vp]),
    "emc_search_set_profiling": (_i, [_vp, _i]),
    "emc_search_timings": (_i, [_vp, _pd, C.POINTER(C.c_long), C.POINTER(C.c_long), C.POINTER(C.c_long), _i]),
    "emc_search_set_planes": (_i, [_vp, _i, _i]),
    "emc_search_get_planes": (_i, [_vp, _i, _i, _pi, _pf]),
    "emc_search_set_overlap": (_i, [_vp, _i]),
    "emc_search_status": (_i, [_vp, _vp]),
    "emc_search_test_wait": (_i, [_vp, C.c_longlong, C.c_uint]),
    "emc_search_plain_noalloc": (_i, [_vp, _vp, _i, _vp, _d, _pd, _pf, _pd, _i, _i, _i, _vp, _vp, _vp, _vp]),
    "emc_cc_adjoint_batch": (_i, [_vp, _i, _pi, C.POINTER(_vp), _pd, _pd, _pd, _i, _pd, _pd, _vp]),
    "emc_cc_adjoint": (_i, [_vp, _i, _vp, _d, _pd, _pd, _i, _pd, _pd, _vp]),
    "emc_tsearch_create": (_i, [_vp, _i, _i, _i, C.POINTER(_vp), _vp]),
    "emc_tsearch_run": (_i, [_vp, _vp, _i, _pd, _i, _vp, _vp, _vp]),
    "emc_tsearch_destroy": (_i, [_vp]),
    "emc_tsearch_peaks": (_i, [_vp, _vp, _i, _i, _i, _pf, _i, _f, _pd, _i, _i, _i, _f, _f, _pd, _pi, _vp]),
    "emc_moving_average": (_i, [_vp, _i, _i, _i, _i, _vp, _vp]),
    "emc_local_normalize": (_i, [_vp, _i, _i, _i, _i, _vp]),
    "emc_symmetry_matrices": (_i, [C.c_char_p, _pd, _pi]),
    "emc_average_create": (_i, [_i, _vp, _f, _i, _pd, _i, _i, C.POINTER(_vp), _vp]),
    "emc_average_add": (_i, [_vp, _vp, _i, _pd, _pf, _pf, _pi, _vp, _i, _pi, _pi, _vp]),
    "emc_average_result": (_i, [_vp, _i, _vp, _vp, C.POINTER(C.c_long), _vp]),
    "emc_average_reset": (_i, [_vp, _vp]),
    "emc_average_boxes": (_i, [_vp, _pi, _pi]),
    "emc_average_destroy": (_i, [_vp]),
    "emc_sf3d_particles": (_i, [C.POINTER(C.c_uint), _d, _pd, _i, _i, _pd, _pd, _i, _vp, _vp]),
    "emc_mrc_read_header": (_i, [C.c_char_p, C.POINTER(MrcHeader)]),
    "emc_mrc_read": (_i, [C.c_char_p, _pi, _pf]),
    "emc_mrc_read_device": (_i, [C.c_char_p, _pi, _vp, _vp]),
    "emc_mrc_write": (_i, [C.c_char_p, _pf, _i, _i, _i, _pf, _pf]),
    "emc_tlt_read": (_i, [C.c_char_p, _pd, _i, _pi, _pi]),
    "emc_window_bounds": (_i, [_pi, _pi, _d, _pd, _pi, _pi, _pi, _pd, _pi]),
    "emc_extract_windows": (_i, [_vp, _i, _i, _i, _pi, _pd, _i, _d, _vp, _pd, _pi, _vp]),
}

_lib = None


def load():
    """Loads libemc_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libemc_b200.so not built: run `python -m emclarity_b200.build` (%s)" % LIB_PATH)
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status, where):
    if status != EMC_OK:
        lib = load()
        raise EmcError(status, where, lib.emc_last_error().decode(errors="replace"))


def call(name, *args):
    lib = load()
    st = getattr(lib, name)(*args)
    check(st, name)
    return st
