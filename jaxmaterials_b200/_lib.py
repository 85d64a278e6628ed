"""ctypes bindings of ``liblippmannschwinger.so`` (declarations in
``include/lippmann_schwinger.h`` and ``include/spectral_net.h``) and of the host library
``libfibres.so`` (``include/fibres.h``).

The library is looked up next to this file first, then through the dynamic loader
(``LD_LIBRARY_PATH``), as the reference wrapper does
(``src/jaxmaterials/solver/lippmann_schwinger.py:284-290``). A missing library is an
error: there is no fallback implementation.
"""

import ctypes
import os
import threading

LIB_NAME = "liblippmannschwinger.so"
_HERE = os.path.dirname(os.path.abspath(__file__))
_lock = threading.Lock()
_lib = None

c_float_p = ctypes.POINTER(ctypes.c_float)
c_int_p = ctypes.POINTER(ctypes.c_int)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_void_p = ctypes.c_void_p

# name -> (restype, argtypes)
SIGNATURES = {
    "lippmann_schwinger_solve": (ctypes.c_int, [c_float_p, c_float_p, c_float_p, c_float_p,
                                                c_float_p, c_int_p, c_float_p, ctypes.c_float,
                                                ctypes.c_float, ctypes.c_int, ctypes.c_int]),
    "lippmann_schwinger_release": (None, []),
    "lsb_create": (ctypes.c_int, [ctypes.POINTER(c_void_p), c_int_p, c_double_p, ctypes.c_int,
                                  ctypes.c_int]),
    "lsb_destroy": (None, [c_void_p]),
    "lsb_set_stream": (ctypes.c_int, [c_void_p, c_void_p]),
    "lsb_solve": (ctypes.c_int, [c_void_p, ctypes.c_int, c_void_p, c_void_p, c_float_p,
                                 c_void_p, c_void_p, c_void_p, c_double_p, ctypes.c_float,
                                 ctypes.c_float, ctypes.c_int, ctypes.c_int, c_int_p, c_int_p,
                                 c_double_p]),
    "lsb_set_precision": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int]),
    "lsb_set_lame_group": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "lsb_set_graphs": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "lsb_set_device_loop": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "lsb_y_variant": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "lsb_set_warm_history": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "lsb_tile_variant": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "lsb_set_tiled": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "lsb_set_slab": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "lsb_pass_config": (ctypes.c_int, [c_void_p, c_int_p]),
    "lsb_set_reference_e0": (ctypes.c_int, [c_void_p, ctypes.c_int, c_double_p]),
    "lsb_c_eff_batch": (ctypes.c_int, [ctypes.c_int, c_int_p, c_double_p,
                                       ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p),
                                       ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                       ctypes.c_float, ctypes.c_int, ctypes.c_double,
                                       c_double_p, c_int_p, c_int_p]),
    "lsb_solve_f64": (ctypes.c_int, [c_void_p, ctypes.c_int, c_void_p, c_void_p, c_double_p,
                                     c_void_p, c_void_p, c_void_p, c_double_p, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_int, ctypes.c_int, c_int_p,
                                     c_int_p, c_double_p]),
    "lsb_history": (ctypes.c_int, [c_void_p, c_double_p, ctypes.c_int]),
    "lsb_kernel_launches": (ctypes.c_longlong, [c_void_p]),
    "lsb_fp64_iters": (ctypes.c_int, [c_void_p, c_int_p]),
    "lsb_profile_step": (ctypes.c_int, [c_void_p, ctypes.c_int, c_void_p, c_void_p, c_void_p,
                                        ctypes.c_int, c_float_p, ctypes.c_int, ctypes.c_char_p,
                                        ctypes.c_int]),
    "lsb_c_eff": (ctypes.c_int, [c_float_p, c_float_p, c_int_p, c_double_p, ctypes.c_float,
                                 ctypes.c_float, ctypes.c_int, ctypes.c_int, c_double_p,
                                 c_int_p]),
    "lsb_solve_noalloc": (ctypes.c_int, [c_int_p, c_double_p, ctypes.c_int, c_void_p, c_void_p,
                                         c_float_p, c_void_p, c_void_p, c_double_p,
                                         ctypes.c_float, ctypes.c_float, ctypes.c_int, c_int_p,
                                         c_int_p, c_double_p, c_void_p]),
    "lsb_ceff_gradient": (ctypes.c_int, [c_int_p, c_void_p, c_double_p, c_void_p, c_void_p,
                                         c_void_p]),
    "lsb_ceff_gradient_f64": (ctypes.c_int, [c_int_p, c_void_p, c_double_p, c_void_p, c_void_p,
                                             c_void_p]),
    "lsb_last_error": (ctypes.c_char_p, []),
    # include/spectral_net.h
    "lsn_pointwise_forward": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_longlong, c_void_p, c_void_p, c_void_p,
                                             c_void_p, c_void_p, c_void_p, ctypes.c_int,
                                             c_void_p]),
    "lsn_pointwise_backward": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_longlong, c_void_p, c_void_p, c_void_p,
                                              c_void_p, ctypes.c_int, c_void_p, c_void_p,
                                              c_void_p, c_void_p, c_void_p]),
    "lsn_spectral_forward": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, c_int_p,
                                            c_int_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "lsn_spectral_backward": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, c_int_p,
                                             c_int_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                             c_void_p, c_void_p]),
    "lsn_truncated_forward": (ctypes.c_int, [ctypes.c_int, c_int_p, c_int_p, c_void_p, c_void_p,
                                             c_void_p, ctypes.c_float, ctypes.c_float, c_void_p]),
    "lsn_truncated_inverse": (ctypes.c_int, [ctypes.c_int, c_int_p, c_int_p, c_void_p, c_void_p,
                                             c_void_p, ctypes.c_float, ctypes.c_float, c_void_p]),
    "lsn_adam": (ctypes.c_int, [ctypes.c_longlong, c_void_p, c_void_p, c_void_p, c_void_p,
                                ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                ctypes.c_int, c_void_p]),
    "lsn_last_error": (ctypes.c_char_p, []),
    "lsb_version": (ctypes.c_int, []),
    "lsb_set_damage": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, ctypes.c_double]),
    "lsb_damage_stress": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_int, c_void_p, c_void_p,
                                         c_void_p, c_void_p, ctypes.c_double, c_void_p,
                                         ctypes.c_int, c_void_p]),
    "lsb_strain_energy": (ctypes.c_int, [ctypes.c_longlong, c_void_p, c_void_p, c_void_p,
                                         c_void_p, c_void_p, ctypes.c_int, c_void_p]),
    "lsb_phase_field_solve": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                             ctypes.c_int, c_int_p, c_double_p]),
    "lsb_set_anisotropic": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, c_double_p]),
    "lsb_voxelise_fibres": (ctypes.c_int, [ctypes.c_int, c_int_p, c_double_p, ctypes.c_double,
                                           ctypes.c_double, c_double_p, c_int_p, c_double_p,
                                           ctypes.c_int, c_void_p, c_void_p]),
}

FIBRES_NAME = "libfibres.so"
c_uint_p = ctypes.POINTER(ctypes.c_uint)
FIBRES_SIGNATURES = {
    "dist_periodic": (None, [ctypes.c_uint, c_double_p, c_double_p, c_double_p, c_double_p]),
    "initialise_rng": (None, [ctypes.c_uint, c_uint_p, ctypes.c_char_p]),
    "move_fibres": (None, [ctypes.c_uint, c_double_p, c_double_p, c_double_p, ctypes.c_uint,
                           ctypes.c_double, ctypes.c_uint, c_uint_p, ctypes.c_char_p]),
    "fibres_move_batch": (ctypes.c_int, [ctypes.c_int, c_uint_p, c_double_p, c_double_p,
                                         c_double_p, ctypes.c_uint, ctypes.c_double,
                                         ctypes.c_uint, ctypes.c_uint, ctypes.c_uint,
                                         ctypes.c_int]),
}
_fibres = None


class LibraryError(RuntimeError):
    pass


def library_path():
    return os.path.join(_HERE, LIB_NAME)


def load():
    """Load the library once and attach the signatures; raise if it is missing."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = library_path()
        try:
            lib = ctypes.CDLL(path if os.path.exists(path) else LIB_NAME)
        except OSError as exc:
            raise LibraryError(
                f"Unable to load {LIB_NAME}: build it with `make -C jaxmaterials_b200/csrc` "
                "(or __graft_entry__.build()) or put it on LD_LIBRARY_PATH.") from exc
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def load_fibres():
    """Load libfibres.so (next to this file, else through the dynamic loader); raise if it
    is missing."""
    global _fibres
    with _lock:
        if _fibres is not None:
            return _fibres
        path = os.path.join(_HERE, FIBRES_NAME)
        try:
            lib = ctypes.CDLL(path if os.path.exists(path) else FIBRES_NAME)
        except OSError as exc:
            raise LibraryError(
                f"Unable to load {FIBRES_NAME}: build it with `make -C jaxmaterials_b200/csrc`."
            ) from exc
        for name, (res, args) in FIBRES_SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _fibres = lib
        return lib


def check_net(rc, what="call"):
    """As check(), for the network kernels of include/spectral_net.h."""
    if rc < 0:
        msg = load().lsn_last_error().decode(errors="replace")
        raise LibraryError(f"{what} failed ({rc}): {msg}")
    return rc


def check(rc, what="call"):
    """Raise on a negative return code, with the library's message."""
    if rc < 0:
        msg = load().lsb_last_error().decode(errors="replace")
        raise LibraryError(f"{what} failed ({rc}): {msg}")
    return rc
