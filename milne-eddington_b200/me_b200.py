"""Python binding of libme_b200.so (the C ABI declared in include/me_b200.h).

A thin ctypes layer: it mirrors the C structures, converts numpy arrays to
pointers and turns negative status codes into exceptions.  All computation
happens in the CUDA library; there is no Python or CPU fallback, and loading
fails loudly if the library has not been built.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libme_b200.so")

ME_MAX_LINES = 20
ME_PATH_LEN = 512
ME_PREC_FP32 = 0
ME_PREC_FP64 = 1

STATUS = {
    0: "ME_OK",
    -1: "ME_ERR_ARG",
    -2: "ME_ERR_CONFIG",
    -3: "ME_ERR_IO",
    -4: "ME_ERR_CUDA",
    -5: "ME_ERR_NODEVICE",
    -6: "ME_ERR_TIMEOUT",
    -7: "ME_ERR_NOMEM",
    -8: "ME_ERR_FORMAT",
}
globals().update({name: code for code, name in STATUS.items()})

_D = ctypes.POINTER(ctypes.c_double)


class MeConfig(ctypes.Structure):
    """struct me_config (include/me_b200.h)."""

    _fields_ = [
        ("nline", ctypes.c_int),
        ("line_lambda0", ctypes.c_double * ME_MAX_LINES),
        ("line_geff", ctypes.c_double * ME_MAX_LINES),
        ("verbose", ctypes.c_int),
        ("num_iter", ctypes.c_int),
        ("num_run", ctypes.c_int),
        ("convg_criteria", ctypes.c_double),
        ("chisq_criteria", ctypes.c_double),
        ("data_path", ctypes.c_char * ME_PATH_LEN),
        ("wavelength_path", ctypes.c_char * ME_PATH_LEN),
        ("weights", ctypes.c_double * 4),
        ("sol_box", ctypes.c_int * 4),
        ("output_fit", ctypes.c_int),
        ("cache_path", ctypes.c_char * ME_PATH_LEN),
        ("result_path", ctypes.c_char * ME_PATH_LEN),
        ("fit_path", ctypes.c_char * ME_PATH_LEN),
        ("damp", ctypes.c_double),
        ("lambda_accept", ctypes.c_double),
        ("lambda_reject", ctypes.c_double),
        ("lambda_limits", ctypes.c_double * 2),
        ("bounds", (ctypes.c_double * 2) * 9),
        ("fixed", ctypes.c_int * 9),
        ("regul", ctypes.c_int * 9),
        ("regul_value", ctypes.c_double * 9),
        ("regul_weight", ctypes.c_double * 9),
        ("regul_any", ctypes.c_int),
        ("vcoeffi", ctypes.c_double),
        ("lcoeffi", ctypes.c_double),
        ("icriteria", ctypes.c_double),
        ("svd_threshold", ctypes.c_double),
        ("hmi_ref", ctypes.c_int),
        ("cache_prof", ctypes.c_int),
        ("nthreads", ctypes.c_int),
        ("nfigures", ctypes.c_int),
        ("step", ctypes.c_double * 9),
        ("nprofiles", ctypes.c_int),
        ("cache_inv", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("rng_seed", ctypes.c_ulonglong),
        ("lines_seen", ctypes.c_int),
        ("data_path_seen", ctypes.c_int),
        ("wavelength_path_seen", ctypes.c_int),
        ("filter_fwhm", ctypes.c_double),
        ("filter_points", ctypes.c_int),
    ]


class MePlanFacts(ctypes.Structure):
    _fields_ = [
        ("nl", ctypes.c_int),
        ("ncut", ctypes.c_int),
        ("ic", ctypes.c_int),
        ("i0", ctypes.c_int),
        ("i1", ctypes.c_int),
        ("npar", ctypes.c_int),
        ("bshift", ctypes.c_double),
        ("limits", (ctypes.c_double * 2) * 9),
        ("fadd_a", ctypes.c_double),
    ]


class MeStats(ctypes.Structure):
    _fields_ = [
        ("pixels", ctypes.c_longlong),
        ("valid", ctypes.c_longlong),
        ("runs", ctypes.c_longlong),
        ("iterations", ctypes.c_longlong),
        ("trials", ctypes.c_longlong),
        ("accepted", ctypes.c_longlong),
        ("syntheses", ctypes.c_longlong),
        ("jacobians", ctypes.c_longlong),
        ("wavelengths", ctypes.c_longlong),
        ("redo_pixels", ctypes.c_longlong),
        ("launches", ctypes.c_longlong),
        ("rounds", ctypes.c_longlong),
        ("kernel_ms", ctypes.c_double),
        ("h2d_ms", ctypes.c_double),
        ("d2h_ms", ctypes.c_double),
        ("init_ms", ctypes.c_double),
        ("learned_done", ctypes.c_longlong),
        ("jac_ms", ctypes.c_double),
        ("svd_ms", ctypes.c_double),
        ("trial_ms", ctypes.c_double),
        ("tail_ms", ctypes.c_double),
        ("tail_trials", ctypes.c_longlong),
        ("tail_jacobians", ctypes.c_longlong),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


# every symbol include/me_b200.h declares
EXPORTED = [
    "me_version", "me_strerror", "me_last_error", "me_config_init", "me_config_parse",
    "me_config_parse_text", "me_plan_create", "me_plan_destroy", "me_plan_get_facts",
    "me_plan_get_carry_chisq", "me_plan_set_carry_chisq", "me_plan_grid", "me_plan_set_grid",
    "me_invert_batch", "me_invert_batch_device", "me_synthesize", "me_synthesize_device",
    "me_synthesize_jacobian", "me_faddeeva", "me_svd", "me_svd_u", "me_init_guess", "me_svd_device", "me_svd_u_device",
    "me_synthesize_jacobian_device", "me_plan_window", "me_plan_set_window",
    "me_invert_batch_device_noalloc", "me_plan_tail_slots", "me_plan_set_tail_slots",
    "me_plan_set_profiling", "me_plan_max_group", "me_plan_set_max_group",
    "me_plan_svd_lanes", "me_plan_set_svd_lanes", "me_plan_set_graphs",
    "me_plan_svd_registers", "me_plan_set_svd_registers", "me_plan_set_feed",
    "me_plan_kernel_variant", "me_plan_set_kernel_variant",
    "me_plan_autotune", "me_plan_last_counters", "me_plan_set_overlap",
    "me_mlp_train_params_default", "me_mlp_train", "me_mlp_destroy", "me_mlp_save",
    "me_mlp_load", "me_mlp_predict", "me_mlp_predict_device", "me_plan_set_initializer",
    "me_mlp_shape", "me_mlp_get_params", "me_mlp_set_params", "me_mlp_loss_grad",
    "me_fits_image_info", "me_fits_read", "me_fits_create", "me_fits_write",
    "me_run_options_default", "me_run", "me_run_config", "me_plan_set_filter",
    "me_mlp_set_gemm", "me_mlp_gemm_launches", "me_gemm_bf16", "me_plan_set_queue_order",
    "me_order_by_key", "me_plan_poll_trace", "me_plan_set_drain", "me_plan_get_drain",
    "me_plan_faddeeva", "me_plan_set_faddeeva", "me_plan_givens", "me_plan_set_givens",
    "me_plan_set_slot_profiles", "me_weideman16", "me_faddeeva_weideman",
]


class MePollRecord(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_double), ("rounds", ctypes.c_longlong),
                ("next", ctypes.c_longlong), ("busy", ctypes.c_int), ("group", ctypes.c_int)]


class MeTuneResult(ctypes.Structure):
    _fields_ = [("window", ctypes.c_int), ("max_group", ctypes.c_int),
                ("tail_slots", ctypes.c_int), ("svd_lanes", ctypes.c_int),
                ("ms", ctypes.c_double), ("trials", ctypes.c_int),
                ("kernel_variant", ctypes.c_int), ("svd_registers", ctypes.c_int),
                ("group_fill", ctypes.c_int), ("drain_poll", ctypes.c_int),
                ("faddeeva", ctypes.c_int), ("slot_profiles", ctypes.c_int)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class MeRunOptions(ctypes.Structure):
    _fields_ = [
        ("ndevices", ctypes.c_int),
        ("devices", ctypes.POINTER(ctypes.c_int)),
        ("batch_pixels", ctypes.c_long),
        ("max_group", ctypes.c_int),
        ("tail_slots", ctypes.c_int),
        ("stop_after_chunks", ctypes.c_long),
        ("initializer", ctypes.c_void_p),
    ]


class MeRunReport(ctypes.Structure):
    _fields_ = [(n, ctypes.c_long) for n in ("nx", "ny", "nw", "counts", "chunk_pixels",
                                             "nchunks", "chunks_done", "chunks_skipped",
                                             "pixels_inverted")] + [("seconds", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class MeMlpTrainParams(ctypes.Structure):
    _fields_ = [
        ("samples", ctypes.c_longlong),
        ("epochs", ctypes.c_int),
        ("batch", ctypes.c_int),
        ("lr", ctypes.c_double),
        ("seed", ctypes.c_ulonglong),
        ("b_range", ctypes.c_double * 2),
        ("cos_theta_range", ctypes.c_double * 2),
        ("phi_range", ctypes.c_double * 2),
        ("v_sigma", ctypes.c_double),
        ("doppler_range", ctypes.c_double * 2),
        ("damping_range", ctypes.c_double * 2),
        ("eta_range", ctypes.c_double * 2),
        ("s", ctypes.c_double),
        ("beta_range", ctypes.c_double * 2),
        ("noise", ctypes.c_double),
        ("gemm", ctypes.c_int),
        ("mix_weight", ctypes.c_double),
        ("mix_b_range", ctypes.c_double * 2),
        ("mix_eta_range", ctypes.c_double * 2),
    ]


class MeError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS.get(status, status)} {detail}".strip())


_lib = None


def lib() -> ctypes.CDLL:
    """Loads libme_b200.so (built by `make -C milne-eddington_b200`)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with make -C {HERE}")
        L = ctypes.CDLL(LIB_PATH)
        L.me_version.restype = ctypes.c_char_p
        L.me_strerror.restype = ctypes.c_char_p
        L.me_last_error.restype = ctypes.c_char_p
        L.me_config_init.argtypes = [ctypes.POINTER(MeConfig)]
        L.me_config_parse.argtypes = [ctypes.c_char_p, ctypes.POINTER(MeConfig), ctypes.c_char_p,
                                      ctypes.c_size_t]
        L.me_config_parse_text.argtypes = [ctypes.c_char_p, ctypes.POINTER(MeConfig),
                                           ctypes.c_char_p, ctypes.c_size_t]
        L.me_plan_create.argtypes = [ctypes.POINTER(MeConfig), _D, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_void_p)]
        L.me_plan_destroy.argtypes = [ctypes.c_void_p]
        L.me_plan_destroy.restype = None
        L.me_plan_get_facts.argtypes = [ctypes.c_void_p, ctypes.POINTER(MePlanFacts)]
        L.me_plan_get_carry_chisq.argtypes = [ctypes.c_void_p]
        L.me_plan_get_carry_chisq.restype = ctypes.c_double
        L.me_plan_set_carry_chisq.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.me_plan_set_carry_chisq.restype = None
        L.me_plan_grid.argtypes = [ctypes.c_void_p]
        L.me_plan_set_grid.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_grid.restype = None
        L.me_plan_window.argtypes = [ctypes.c_void_p]
        L.me_plan_set_window.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_window.restype = None
        L.me_plan_tail_slots.argtypes = [ctypes.c_void_p]
        L.me_plan_set_tail_slots.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_tail_slots.restype = None
        L.me_plan_set_profiling.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_profiling.restype = None
        L.me_plan_max_group.argtypes = [ctypes.c_void_p]
        L.me_plan_set_max_group.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_max_group.restype = None
        L.me_plan_autotune.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long,
                                       ctypes.c_void_p, ctypes.POINTER(MeTuneResult)]
        L.me_plan_last_counters.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint),
                                            ctypes.c_long]
        L.me_plan_set_slot_profiles.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_slot_profiles.restype = None
        L.me_plan_givens.argtypes = [ctypes.c_void_p]
        L.me_plan_givens.restype = ctypes.c_int
        L.me_plan_set_givens.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_givens.restype = None
        L.me_plan_faddeeva.argtypes = [ctypes.c_void_p]
        L.me_plan_faddeeva.restype = ctypes.c_int
        L.me_plan_set_faddeeva.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_faddeeva.restype = None
        L.me_weideman16.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.me_weideman16.restype = None
        L.me_faddeeva_weideman.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.me_faddeeva_weideman.restype = ctypes.c_int
        L.me_plan_set_drain.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.me_plan_set_drain.restype = None
        L.me_plan_get_drain.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int)]
        L.me_plan_get_drain.restype = None
        L.me_plan_poll_trace.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.me_plan_poll_trace.restype = ctypes.c_int
        L.me_plan_set_overlap.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_overlap.restype = None
        L.me_plan_set_queue_order.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_queue_order.restype = None
        L.me_order_by_key.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_ubyte), ctypes.c_long,
                                      ctypes.POINTER(ctypes.c_longlong)]
        L.me_plan_set_graphs.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_graphs.restype = None
        L.me_plan_svd_lanes.argtypes = [ctypes.c_void_p]
        L.me_plan_set_svd_lanes.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_svd_lanes.restype = None
        L.me_plan_kernel_variant.argtypes = [ctypes.c_void_p]
        L.me_plan_set_kernel_variant.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_kernel_variant.restype = None
        L.me_plan_set_feed.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_feed.restype = None
        L.me_plan_svd_registers.argtypes = [ctypes.c_void_p]
        L.me_plan_set_svd_registers.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_plan_set_svd_registers.restype = None
        L.me_invert_batch.argtypes = [ctypes.c_void_p, _D, ctypes.c_long, _D, _D,
                                      ctypes.POINTER(MeStats)]
        L.me_invert_batch_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.POINTER(MeStats)]
        L.me_synthesize.argtypes = [ctypes.c_void_p, _D, ctypes.c_long, _D]
        L.me_synthesize_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long,
                                           ctypes.c_void_p, ctypes.c_void_p]
        L.me_synthesize_jacobian.argtypes = [ctypes.c_void_p, _D, ctypes.c_long, ctypes.c_double,
                                             _D, _D]
        L.me_faddeeva.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, ctypes.c_long, _D, _D,
                                  ctypes.c_int]
        L.me_svd.argtypes = [_D, ctypes.c_long, ctypes.c_int, _D, _D, _D, ctypes.c_int]
        L.me_svd_u.argtypes = [_D, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D,
                               _D, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.me_svd_u_device.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]
        L.me_svd_device.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.me_synthesize_jacobian_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_long, ctypes.c_double,
                                                    ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_void_p]
        L.me_invert_batch_device_noalloc.argtypes = [ctypes.POINTER(MeConfig), _D, ctypes.c_int,
                                                     ctypes.c_void_p, ctypes.c_long,
                                                     ctypes.c_void_p, _D, ctypes.c_void_p]
        L.me_init_guess.argtypes = [ctypes.c_void_p, _D, ctypes.c_long, _D, _D,
                                    ctypes.POINTER(ctypes.c_int)]
        _F = ctypes.POINTER(ctypes.c_float)
        L.me_mlp_train_params_default.argtypes = [ctypes.POINTER(MeMlpTrainParams)]
        L.me_mlp_train.argtypes = [ctypes.c_void_p, ctypes.POINTER(MeMlpTrainParams),
                                   ctypes.POINTER(ctypes.c_void_p), _D]
        L.me_mlp_destroy.argtypes = [ctypes.c_void_p]
        L.me_mlp_destroy.restype = None
        L.me_mlp_save.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.me_mlp_load.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.me_mlp_predict.argtypes = [ctypes.c_void_p, _D, ctypes.c_long, _D]
        L.me_mlp_predict_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long,
                                            ctypes.c_void_p, ctypes.c_void_p]
        L.me_plan_set_initializer.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.me_mlp_shape.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)]
        L.me_mlp_get_params.argtypes = [ctypes.c_void_p, _F]
        L.me_mlp_set_params.argtypes = [ctypes.c_void_p, _F]
        L.me_mlp_loss_grad.argtypes = [ctypes.c_void_p, _F, _F, ctypes.c_int, _D, _F]
        L.me_mlp_set_gemm.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.me_mlp_gemm_launches.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong),
                                           ctypes.POINTER(ctypes.c_longlong)]
        _U16 = ctypes.POINTER(ctypes.c_uint16)
        L.me_gemm_bf16.argtypes = [ctypes.c_int, ctypes.c_int, _U16, _U16, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, _F, ctypes.c_int,
                                   _F, _F, ctypes.POINTER(ctypes.c_int)]
        _L8 = ctypes.c_long * 8
        L.me_fits_image_info.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int), _L8]
        L.me_fits_read.argtypes = [ctypes.c_char_p, ctypes.c_long, ctypes.c_long, _D]
        L.me_fits_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_long)]
        L.me_fits_write.argtypes = [ctypes.c_char_p, ctypes.c_long, ctypes.c_long, _D]
        L.me_plan_set_filter.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_int]
        L.me_run_options_default.argtypes = [ctypes.POINTER(MeRunOptions)]
        L.me_run.argtypes = [ctypes.c_char_p, ctypes.POINTER(MeRunOptions),
                             ctypes.POINTER(MeRunReport)]
        L.me_run_config.argtypes = [ctypes.POINTER(MeConfig), ctypes.POINTER(MeRunOptions),
                                    ctypes.POINTER(MeRunReport)]
        _lib = L
    return _lib


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


def _check(status: int, where: str):
    if status != 0:
        raise MeError(status, where, lib().me_last_error().decode(errors="replace"))


def parse_config_text(text: str) -> MeConfig:
    """me_config_parse_text: the reference's keyword semantics (Src/RINPUT.c:361-563)."""
    cfg = MeConfig()
    err = ctypes.create_string_buffer(512)
    st = lib().me_config_parse_text(text.encode(), ctypes.byref(cfg), err, 512)
    if st != 0:
        raise MeError(st, "me_config_parse_text", err.value.decode(errors="replace"))
    return cfg


def parse_config(path: str) -> MeConfig:
    cfg = MeConfig()
    err = ctypes.create_string_buffer(512)
    st = lib().me_config_parse(path.encode(), ctypes.byref(cfg), err, 512)
    if st != 0:
        raise MeError(st, "me_config_parse", err.value.decode(errors="replace"))
    return cfg


def default_config() -> MeConfig:
    cfg = MeConfig()
    _check(lib().me_config_init(ctypes.byref(cfg)), "me_config_init")
    return cfg


class Plan:
    """me_plan: one wavelength grid + control file on one GPU (INIT_INV)."""

    def __init__(self, cfg: MeConfig, wavelengths: np.ndarray, device: int = 0):
        self.cfg = cfg
        self.wavelengths = np.ascontiguousarray(wavelengths, dtype=np.float64)
        self.nl = int(self.wavelengths.size)
        h = ctypes.c_void_p()
        _check(lib().me_plan_create(ctypes.byref(cfg), _ptr(self.wavelengths), self.nl, device,
                                    ctypes.byref(h)), "me_plan_create")
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().me_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def facts(self) -> dict:
        f = MePlanFacts()
        _check(lib().me_plan_get_facts(self._h, ctypes.byref(f)), "me_plan_get_facts")
        return {"nl": f.nl, "ncut": f.ncut, "ic": f.ic, "i0": f.i0, "i1": f.i1, "npar": f.npar,
                "bshift": f.bshift, "limits": np.array([[f.limits[i][0], f.limits[i][1]]
                                                        for i in range(9)]),
                "fadd_a": f.fadd_a}

    @property
    def carry_chisq(self) -> float:
        return lib().me_plan_get_carry_chisq(self._h)

    @carry_chisq.setter
    def carry_chisq(self, v: float):
        lib().me_plan_set_carry_chisq(self._h, float(v))

    @property
    def grid(self) -> int:
        return lib().me_plan_grid(self._h)

    @grid.setter
    def grid(self, g: int):
        lib().me_plan_set_grid(self._h, int(g))

    @property
    def window(self) -> int:
        return lib().me_plan_window(self._h)

    @window.setter
    def window(self, w: int):
        lib().me_plan_set_window(self._h, int(w))

    @property
    def tail_slots(self) -> int:
        return lib().me_plan_tail_slots(self._h)

    @tail_slots.setter
    def tail_slots(self, n: int):
        lib().me_plan_set_tail_slots(self._h, int(n))

    @property
    def max_group(self) -> int:
        return lib().me_plan_max_group(self._h)

    @max_group.setter
    def max_group(self, lanes: int):
        lib().me_plan_set_max_group(self._h, int(lanes))

    @property
    def svd_lanes(self) -> int:
        return lib().me_plan_svd_lanes(self._h)

    @svd_lanes.setter
    def svd_lanes(self, lanes: int):
        lib().me_plan_set_svd_lanes(self._h, int(lanes))

    @property
    def svd_registers(self) -> int:
        """SVD solves with the 9x9 matrix in registers (all nine parameters free):
        0 shared memory, 1 registers in the full rounds, 2 also after the drain."""
        return lib().me_plan_svd_registers(self._h)

    @svd_registers.setter
    def svd_registers(self, mode: int):
        lib().me_plan_set_svd_registers(self._h, int(mode))

    def set_filter(self, offsets_mA, weights):
        """Instrument filter: offsets [mA] and weights of each observed wavelength's
        sub-wavelengths (one offset removes it)."""
        off = np.ascontiguousarray(offsets_mA, dtype=np.float64)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        assert off.shape == w.shape and off.ndim == 1
        _check(lib().me_plan_set_filter(self._h, _ptr(off), _ptr(w), off.size),
               "me_plan_set_filter")

    def autotune(self, d_prof: int, npix: int, stream: int = 0) -> dict:
        """me_plan_autotune on device profiles; returns the chosen setting."""
        r = MeTuneResult()
        _check(lib().me_plan_autotune(self._h, ctypes.c_void_p(d_prof), npix,
                                      ctypes.c_void_p(stream) if stream else None,
                                      ctypes.byref(r)), "me_plan_autotune")
        return r.as_dict()

    def set_slot_profiles(self, on: bool):
        """Kernels read the observed profiles from a slot-major copy (default off)."""
        lib().me_plan_set_slot_profiles(self._h, int(bool(on)))

    @property
    def givens(self) -> int:
        """FP32 plans' SVD Givens rotations: 1 from one reciprocal square root,
        0 the reference's pythag and division."""
        return lib().me_plan_givens(self._h)

    @givens.setter
    def givens(self, mode: int):
        lib().me_plan_set_givens(self._h, int(mode))

    @property
    def faddeeva(self) -> int:
        """FP32 Faddeeva evaluation: 0 the reference's regions and Alg-916, 1
        Weideman's 16-term series."""
        return lib().me_plan_faddeeva(self._h)

    @faddeeva.setter
    def faddeeva(self, mode: int):
        lib().me_plan_set_faddeeva(self._h, int(mode))

    @property
    def drain(self) -> tuple:
        """(group_fill, poll_rounds) of the rounds after the queue drains."""
        f, r = ctypes.c_int(), ctypes.c_int()
        lib().me_plan_get_drain(self._h, ctypes.byref(f), ctypes.byref(r))
        return f.value, r.value

    @drain.setter
    def drain(self, v):
        lib().me_plan_set_drain(self._h, int(v[0]), int(v[1]))

    def poll_trace(self) -> list:
        """The queue checks of the last batch: dicts of ms (host time since its
        rounds began), rounds, next (queue position), busy (pixels in flight)
        and group (lanes per pixel; 0 = tail kernel launched, -1 = first pass
        ended)."""
        n = lib().me_plan_poll_trace(self._h, None, 0)
        buf = (MePollRecord * max(n, 1))()
        n = lib().me_plan_poll_trace(self._h, buf, n)
        return [{k: getattr(buf[i], k) for k, _ in MePollRecord._fields_} for i in range(n)]

    def last_counters(self, npix: int) -> np.ndarray:
        """[npix][4] runs, iterations, trials, accepted of the last batch."""
        out = np.zeros((npix, 4), dtype=np.uint32)
        _check(lib().me_plan_last_counters(self._h, out.ctypes.data_as(
            ctypes.POINTER(ctypes.c_uint)), npix), "me_plan_last_counters")
        return out

    @property
    def kernel_variant(self) -> int:
        """Jacobian / trial kernel variant: 0 default, 1 / 2 = 64 / 256 pixels per
        CTA, 3 = grid staged in shared memory, 4 = no Faddeeva reciprocal table,
        5 = normal-equation sums in shared memory (FP32)."""
        return lib().me_plan_kernel_variant(self._h)

    @kernel_variant.setter
    def kernel_variant(self, v: int):
        lib().me_plan_set_kernel_variant(self._h, int(v))

    def set_feed(self, mode=True):
        """me_invert_batch from page-locked host memory: copy the map in chunks
        and start inverting as they land (True / 1, default); 2: the same without
        the global re-sort of the queue's untaken part; False / 0: copy it whole."""
        lib().me_plan_set_feed(self._h, int(mode))

    def set_overlap(self, on: bool = True):
        """Later-trial SVDs on a second stream beside the Jacobian kernel (default on)."""
        lib().me_plan_set_overlap(self._h, int(bool(on)))

    def set_queue_order(self, on: bool = True):
        """With a learned start, queue pixels by descending misfit of their start
        (default on); off: pixel order."""
        lib().me_plan_set_queue_order(self._h, int(bool(on)))

    def set_graphs(self, on: bool = True):
        """Rounds between queue checks as one CUDA graph launch (default on)."""
        lib().me_plan_set_graphs(self._h, int(bool(on)))

    def set_profiling(self, on: bool = True):
        """Per-kernel device time in the stats (CUDA events around every launch)."""
        lib().me_plan_set_profiling(self._h, int(bool(on)))

    def set_initializer(self, init: Optional["Initializer"]):
        """Attaches a learned initialiser (None detaches); the plan does not own it."""
        _check(lib().me_plan_set_initializer(self._h, init.handle if init is not None else None),
               "me_plan_set_initializer")
        self._init = init

    def invert(self, prof: np.ndarray, want_fit: bool = False, out: Optional[np.ndarray] = None):
        """me_invert_batch on host arrays: prof [npix][4][nl] -> res [npix][10] (+fit).
        out (optional): a C-contiguous float64 [npix][10] array for the results,
        e.g. a view of pinned host memory."""
        prof = np.ascontiguousarray(prof, dtype=np.float64)
        npix = prof.shape[0]
        assert prof.shape[1:] == (4, self.nl)
        if out is not None:
            assert out.shape == (npix, 10) and out.dtype == np.float64 and out.flags["C_CONTIGUOUS"]
            res = out
        else:
            res = np.zeros((npix, 10))
        fit = np.zeros((npix, 4, self.nl)) if want_fit else None
        st = MeStats()
        _check(lib().me_invert_batch(self._h, _ptr(prof), npix, _ptr(res), _ptr(fit),
                                     ctypes.byref(st)), "me_invert_batch")
        return (res, fit, st.as_dict()) if want_fit else (res, st.as_dict())

    def invert_device(self, d_prof: int, npix: int, d_res: int, d_fit: int = 0, stream: int = 0):
        """me_invert_batch_device on raw device pointers (e.g. torch tensor .data_ptr())."""
        st = MeStats()
        _check(lib().me_invert_batch_device(self._h, ctypes.c_void_p(d_prof), npix,
                                            ctypes.c_void_p(d_res),
                                            ctypes.c_void_p(d_fit) if d_fit else None,
                                            ctypes.c_void_p(stream) if stream else None,
                                            ctypes.byref(st)), "me_invert_batch_device")
        return st.as_dict()

    def synthesize(self, par: np.ndarray) -> np.ndarray:
        par = np.ascontiguousarray(par, dtype=np.float64).reshape(-1, 9)
        out = np.zeros((par.shape[0], 4, self.nl))
        _check(lib().me_synthesize(self._h, _ptr(par), par.shape[0], _ptr(out)), "me_synthesize")
        return out

    def synthesize_device(self, d_par: int, npix: int, d_prof: int, stream: int = 0):
        _check(lib().me_synthesize_device(self._h, ctypes.c_void_p(d_par), npix,
                                          ctypes.c_void_p(d_prof),
                                          ctypes.c_void_p(stream) if stream else None),
               "me_synthesize_device")

    def synthesize_jacobian_device(self, d_par: int, npix: int, step7: float, d_prof: int,
                                   d_jac: int, stream: int = 0):
        _check(lib().me_synthesize_jacobian_device(self._h, ctypes.c_void_p(d_par), npix,
                                                   float(step7), ctypes.c_void_p(d_prof),
                                                   ctypes.c_void_p(d_jac) if d_jac else None,
                                                   ctypes.c_void_p(stream) if stream else None),
               "me_synthesize_jacobian_device")

    def synthesize_jacobian(self, par: np.ndarray, step7: float):
        par = np.ascontiguousarray(par, dtype=np.float64).reshape(-1, 9)
        n = par.shape[0]
        prof = np.zeros((n, 4, self.nl))
        jac = np.zeros((n, 4, 9, self.nl))
        _check(lib().me_synthesize_jacobian(self._h, _ptr(par), n, float(step7), _ptr(prof),
                                            _ptr(jac)), "me_synthesize_jacobian")
        return prof, jac

    def init_guess(self, prof: np.ndarray):
        prof = np.ascontiguousarray(prof, dtype=np.float64)
        n = prof.shape[0]
        guess = np.zeros((n, 9))
        extra = np.zeros((n, 5))
        status = np.zeros(n, dtype=np.int32)
        _check(lib().me_init_guess(self._h, _ptr(prof), n, _ptr(guess), _ptr(extra),
                                   status.ctypes.data_as(ctypes.POINTER(ctypes.c_int))),
               "me_init_guess")
        return guess, extra, status


def faddeeva(nfigures: int, nu: np.ndarray, a: np.ndarray, precision: int = ME_PREC_FP64,
             device: int = 0):
    nu = np.ascontiguousarray(nu, dtype=np.float64).ravel()
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    H = np.zeros_like(nu)
    L = np.zeros_like(nu)
    _check(lib().me_faddeeva(nfigures, precision, _ptr(nu), _ptr(a), nu.size, _ptr(H), _ptr(L),
                             device), "me_faddeeva")
    return H, L


def faddeeva_weideman(nu: np.ndarray, a: np.ndarray, device: int = 0):
    """w(nu + i a) by Weideman's 16-term series in FP32 on the device: (H, L)."""
    nu = np.ascontiguousarray(nu, dtype=np.float64).ravel()
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    H = np.zeros_like(nu)
    L = np.zeros_like(nu)
    _check(lib().me_faddeeva_weideman(_ptr(nu), _ptr(a), nu.size, _ptr(H), _ptr(L), device),
           "me_faddeeva_weideman")
    return H, L


def weideman16():
    """(c_0..c_15, L) of the FP32 Weideman series the library evaluates."""
    c = np.zeros(16, dtype=np.float32)
    L = ctypes.c_float()
    lib().me_weideman16(c.ctypes.data_as(ctypes.c_void_p), ctypes.byref(L))
    return c, L.value


def invert_device_noalloc(cfg: MeConfig, wavelengths: np.ndarray, d_prof: int, npix: int,
                          d_res: int, carry_chisq: float = 0.0, stream: int = 0) -> float:
    """me_invert_batch_device_noalloc: the inversion with no device allocation
    (fixed static scratch, at most ME_NOALLOC_MAX_PIXELS = 65536 pixels per
    call).  Returns the LM chi^2 to carry into the next call of the same map."""
    lam = np.ascontiguousarray(wavelengths, dtype=np.float64)
    carry = np.array([carry_chisq], dtype=np.float64)
    _check(lib().me_invert_batch_device_noalloc(ctypes.byref(cfg), _ptr(lam), lam.size,
                                                ctypes.c_void_p(d_prof), npix,
                                                ctypes.c_void_p(d_res), _ptr(carry),
                                                ctypes.c_void_p(stream) if stream else None),
           "me_invert_batch_device_noalloc")
    return float(carry[0])


def svd_device(d_a: int, nmat: int, n: int, d_u: int, d_w: int, d_v: int, stream: int = 0):
    _check(lib().me_svd_device(ctypes.c_void_p(d_a), nmat, n, ctypes.c_void_p(d_u),
                               ctypes.c_void_p(d_w), ctypes.c_void_p(d_v),
                               ctypes.c_void_p(stream) if stream else None), "me_svd_device")


def svd(a: np.ndarray, device: int = 0):
    a = np.ascontiguousarray(a, dtype=np.float64)
    nmat, n, _ = a.shape
    u = np.zeros_like(a)
    v = np.zeros_like(a)
    w = np.zeros((nmat, n))
    _check(lib().me_svd(_ptr(a), nmat, n, _ptr(u), _ptr(w), _ptr(v), device), "me_svd")
    return u, w, v


def svd_u_device(d_a: int, nmat: int, n: int, d_u: int, d_w: int, lanes: int = 1,
                 fast: bool = False, stream: int = 0):
    _check(lib().me_svd_u_device(ctypes.c_void_p(d_a), nmat, n, lanes, 1 if fast else 0,
                                 ctypes.c_void_p(d_u), ctypes.c_void_p(d_w),
                                 ctypes.c_void_p(stream) if stream else None), "me_svd_u_device")


def svd_u(a: np.ndarray, lanes: int = 1, fast: bool = False, device: int = 0):
    """U and w of the inversion's trial-step decomposition (no V) of each
    n x n matrix of a [nmat, n, n], with `lanes` lanes per matrix and the
    Givens rotations' fast form (FP32 plans) or the reference's; returns
    (u, w, number of matrices that hit the 50-sweep limit)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    nmat, n, _ = a.shape
    u = np.zeros_like(a)
    w = np.zeros((nmat, n))
    hits = ctypes.c_int(0)
    _check(lib().me_svd_u(_ptr(a), nmat, n, lanes, 1 if fast else 0, _ptr(u), _ptr(w),
                          ctypes.byref(hits), device), "me_svd_u")
    return u, w, hits.value


def _fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def mlp_train_params(**overrides) -> MeMlpTrainParams:
    """me_mlp_train_params_default with keyword overrides (ranges as 2-tuples)."""
    tp = MeMlpTrainParams()
    _check(lib().me_mlp_train_params_default(ctypes.byref(tp)), "me_mlp_train_params_default")
    for k, v in overrides.items():
        if not hasattr(tp, k):
            raise KeyError(k)
        if isinstance(v, (tuple, list)):
            arr = getattr(tp, k)
            arr[0], arr[1] = float(v[0]), float(v[1])
        else:
            setattr(tp, k, v)
    return tp


class Initializer:
    """me_mlp: the learned initialiser (4 nl -> 256 -> 256 -> 256 -> 10 GELU MLP)."""

    def __init__(self, handle: ctypes.c_void_p, final_loss: float = float("nan")):
        self._h = handle
        self.final_loss = final_loss

    @classmethod
    def train(cls, plan: "Plan", params: Optional[MeMlpTrainParams] = None, **overrides):
        tp = params if params is not None else mlp_train_params(**overrides)
        h = ctypes.c_void_p()
        loss = np.zeros(1)
        _check(lib().me_mlp_train(plan.handle, ctypes.byref(tp), ctypes.byref(h), _ptr(loss)),
               "me_mlp_train")
        return cls(h, float(loss[0]))

    @classmethod
    def load(cls, path: str, device: int = 0):
        h = ctypes.c_void_p()
        _check(lib().me_mlp_load(str(path).encode(), device, ctypes.byref(h)), "me_mlp_load")
        return cls(h)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().me_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def save(self, path: str):
        _check(lib().me_mlp_save(self._h, str(path).encode()), "me_mlp_save")

    def shape(self):
        nl, nip, npar = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        _check(lib().me_mlp_shape(self._h, ctypes.byref(nl), ctypes.byref(nip),
                                  ctypes.byref(npar)), "me_mlp_shape")
        return nl.value, nip.value, npar.value

    def predict(self, prof: np.ndarray) -> np.ndarray:
        prof = np.ascontiguousarray(prof, dtype=np.float64)
        par = np.zeros((prof.shape[0], 9))
        _check(lib().me_mlp_predict(self._h, _ptr(prof), prof.shape[0], _ptr(par)),
               "me_mlp_predict")
        return par

    def predict_device(self, d_prof: int, npix: int, d_par: int, stream: int = 0):
        _check(lib().me_mlp_predict_device(self._h, ctypes.c_void_p(d_prof), npix,
                                           ctypes.c_void_p(d_par), ctypes.c_void_p(stream)),
               "me_mlp_predict_device")

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.shape()[2], dtype=np.float32)
        _check(lib().me_mlp_get_params(self._h, _fptr(out)), "me_mlp_get_params")
        return out

    def set_params(self, params: np.ndarray):
        params = np.ascontiguousarray(params, dtype=np.float32)
        assert params.size == self.shape()[2]
        _check(lib().me_mlp_set_params(self._h, _fptr(params)), "me_mlp_set_params")

    def loss_grad(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = np.zeros(1)
        grad = np.zeros(self.shape()[2], dtype=np.float32)
        _check(lib().me_mlp_loss_grad(self._h, _fptr(x), _fptr(t), x.shape[0], _ptr(loss),
                                      _fptr(grad)), "me_mlp_loss_grad")
        return float(loss[0]), grad

    def set_gemm(self, path: str):
        """"tcgen05" (the default) or "mma_sync": the GEMM kernel of training and
        inference."""
        _check(lib().me_mlp_set_gemm(self._h, GEMM_PATHS[path]), "me_mlp_set_gemm")

    def gemm_launches(self):
        """{"tcgen05": n, "mma_sync": n}: GEMM launches of each kernel so far."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        _check(lib().me_mlp_gemm_launches(self._h, ctypes.byref(a), ctypes.byref(b)),
               "me_mlp_gemm_launches")
        return {"tcgen05": a.value, "mma_sync": b.value}


GEMM_PATHS = {"tcgen05": 0, "mma_sync": 1}


def order_by_key(keys: np.ndarray, device: int = 0) -> np.ndarray:
    """The queue order's stable counting sort on the GPU: indices of keys
    (uint8, each < 128) by ascending key, equal keys in index order."""
    keys = np.ascontiguousarray(keys, dtype=np.uint8)
    out = np.zeros(keys.size, dtype=np.int64)
    _check(lib().me_order_by_key(device, keys.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                                 keys.size, out.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))),
           "me_order_by_key")
    return out


def gemm_bf16(a: np.ndarray, bt: np.ndarray, path: str = "tcgen05", split: int = 1,
              bias: Optional[np.ndarray] = None, gelu: bool = False, device: int = 0):
    """One GEMM of the initialiser's kernels: a [m][r] and bt [n][r] are BF16
    bit patterns (uint16); returns (z, y, kernel that ran) with z = a bt^T +
    bias and y = GELU(z) or z (FP32; z is None for split > 1)."""
    a = np.ascontiguousarray(a, dtype=np.uint16)
    bt = np.ascontiguousarray(bt, dtype=np.uint16)
    m, r = a.shape
    n = bt.shape[0]
    assert bt.shape[1] == r
    y = np.zeros((m, n), dtype=np.float32)
    z = np.zeros((m, n), dtype=np.float32) if split == 1 else None
    b = None if bias is None else np.ascontiguousarray(bias, dtype=np.float32)
    ran = ctypes.c_int(-1)
    u16 = ctypes.POINTER(ctypes.c_uint16)
    _check(lib().me_gemm_bf16(device, GEMM_PATHS[path], a.ctypes.data_as(u16),
                              bt.ctypes.data_as(u16), m, n, r, split,
                              None if b is None else _fptr(b), int(gelu),
                              None if z is None else _fptr(z), _fptr(y), ctypes.byref(ran)),
           "me_gemm_bf16")
    names = {v: k for k, v in GEMM_PATHS.items()}
    return z, y, names[ran.value]


# ---------------------------------------------------------------------------
# FITS primary-HDU I/O and the driver
# ---------------------------------------------------------------------------
def fits_info(path):
    """(bitpix, shape in FITS order NAXIS1, NAXIS2, ...)."""
    b, n = ctypes.c_int(), ctypes.c_int()
    ax = (ctypes.c_long * 8)()
    _check(lib().me_fits_image_info(str(path).encode(), ctypes.byref(b), ctypes.byref(n), ax),
           "me_fits_image_info")
    return b.value, tuple(ax[i] for i in range(n.value))


def fits_read(path, first: int = 0, n: int = -1) -> np.ndarray:
    """Elements [first, first + n) of the primary array as doubles (FITS order)."""
    _, shape = fits_info(path)
    total = int(np.prod(shape)) if shape else 0
    if n < 0:
        n = total - first
    out = np.zeros(n)
    _check(lib().me_fits_read(str(path).encode(), first, n, _ptr(out)), "me_fits_read")
    return out


def fits_create(path, shape):
    """Zero-filled BITPIX -64 image; shape in FITS order (NAXIS1 first)."""
    ax = (ctypes.c_long * len(shape))(*shape)
    _check(lib().me_fits_create(str(path).encode(), len(shape), ax), "me_fits_create")


def fits_write(path, first: int, values: np.ndarray):
    v = np.ascontiguousarray(values, dtype=np.float64).ravel()
    _check(lib().me_fits_write(str(path).encode(), first, v.size, _ptr(v)), "me_fits_write")


def run_options(**kw) -> MeRunOptions:
    o = MeRunOptions()
    _check(lib().me_run_options_default(ctypes.byref(o)), "me_run_options_default")
    devices = kw.pop("devices", None)
    init = kw.pop("initializer", None)
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    if devices is not None:
        arr = (ctypes.c_int * len(devices))(*devices)
        o.devices = arr
        o.ndevices = len(devices)
        o._devices_keepalive = arr
    if init is not None:
        o.initializer = init.handle.value if hasattr(init.handle, "value") else init.handle
    return o


def run(ctl_path, **kw) -> dict:
    """me_run: the driver on a control file; returns the run report."""
    o = run_options(**kw)
    rep = MeRunReport()
    _check(lib().me_run(str(ctl_path).encode(), ctypes.byref(o), ctypes.byref(rep)), "me_run")
    return rep.as_dict()
