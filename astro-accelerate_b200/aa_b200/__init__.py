"""Python binding of the B200-native dedispersion library (libaa_b200.so).

The classes mirror the reference's ctypes wrapper of its C ABI
(AstroAccelerate v1.3.1, cmake/py_astro_accelerate.py.in:120-560):
``aa_py_filterbank_metadata``, ``aa_py_dm``, ``aa_py_ddtr_plan``,
``aa_py_pipeline_components``, ``aa_py_pipeline_component_options`` and
``aa_py_pipeline`` keep their names, arguments and return values, so a script
written against the reference runs against this library.  The functions below
them expose the library's own seam (stateless device-pointer entry points)
and extensions.

There is no CPU fallback: every entry point runs the CUDA kernels of
libaa_b200.so and fails loudly when the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libaa_b200.so")

FLOAT = ctypes.c_float
PFLOAT = ctypes.POINTER(FLOAT)
PPFLOAT = ctypes.POINTER(PFLOAT)
PPPFLOAT = ctypes.POINTER(PPFLOAT)

KIND_SHARED8, KIND_SHARED16, KIND_SHARED4, KIND_CACHE = 0, 1, 2, 3
KIND_NAMES = {0: "shared8", 1: "shared16", 2: "shared4", 3: "cache"}
STRIDE_REFERENCE, STRIDE_TRUE = 0, 1
STATUS_ERROR, STATUS_FINISHED, STATUS_HAS_MORE, STATUS_FINISHED_COMPONENT = -1, 0, 1, 2


def build(jobs: int = 8) -> str:
    """Compile libaa_b200.so for sm_100a with nvcc (no GPU needed)."""
    subprocess.check_call(["make", "-C", PKG_ROOT, f"-j{jobs}"], stdout=subprocess.DEVNULL)
    return LIB_PATH


class filterbank_metadata_struct(ctypes.Structure):
    """include/aa_py_filterbank_metadata.hpp:15-25."""

    _fields_ = [("m_tstart", ctypes.c_double), ("m_tsamp", ctypes.c_double), ("m_fch1", ctypes.c_double),
                ("m_foff", ctypes.c_double), ("m_nbits", ctypes.c_int), ("m_nsamples", ctypes.c_int),
                ("m_nchans", ctypes.c_int), ("m_src_raj", ctypes.c_double)]


class sigproc_header_struct(ctypes.Structure):
    """aa_b200_sigproc_header_struct (include/aa_b200.h)."""
    _fields_ = [("telescope_id", ctypes.c_int), ("machine_id", ctypes.c_int), ("data_type", ctypes.c_int),
                ("barycentric", ctypes.c_int), ("pulsarcentric", ctypes.c_int), ("az_start", ctypes.c_double),
                ("za_start", ctypes.c_double), ("src_raj", ctypes.c_double), ("src_dej", ctypes.c_double),
                ("tstart", ctypes.c_double), ("tsamp", ctypes.c_double), ("nbits", ctypes.c_int),
                ("nsamples_keyword", ctypes.c_int), ("nchans", ctypes.c_int), ("nifs", ctypes.c_int),
                ("fch1", ctypes.c_double), ("foff", ctypes.c_double), ("fchannel", ctypes.c_double),
                ("refdm", ctypes.c_double), ("period", ctypes.c_double), ("data_start", ctypes.c_longlong),
                ("data_bytes", ctypes.c_longlong), ("nsamp", ctypes.c_longlong)]


class aa_py_pipeline_components(ctypes.Structure):
    """include/aa_py_pipeline_api.hpp:20-25."""

    _fields_ = [("dedispersion", ctypes.c_bool), ("analysis", ctypes.c_bool), ("periodicity", ctypes.c_bool),
                ("fdas", ctypes.c_bool)]


class aa_py_pipeline_component_options(ctypes.Structure):
    """include/aa_py_pipeline_api.hpp:32-48."""

    _fields_ = [(n, ctypes.c_bool) for n in (
        "zero_dm", "zero_dm_with_outliers", "input_DDTR_normalization", "output_DDTR_normalization",
        "set_bandpass_average", "old_rfi", "copy_ddtr_data_to_host", "msd_baseline_noise", "output_dmt",
        "output_ffdot_plan", "output_fdas_list", "candidate_algorithm", "fdas_custom_fft", "fdas_inbin",
        "fdas_norm")]


class aa_b200_dm(ctypes.Structure):
    """include/aa_ddtr_plan.hpp:28-34 struct dm."""

    _fields_ = [("low", ctypes.c_float), ("high", ctypes.c_float), ("step", ctypes.c_float),
                ("inBin", ctypes.c_int), ("outBin", ctypes.c_int)]


_lib = None


def lib():
    """The loaded libaa_b200.so with its prototypes (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libaa_b200.so is not built ({LIB_PATH}); run aa_b200.build() or "
                           "`make -C astro-accelerate_b200`")
    L = ctypes.CDLL(LIB_PATH)
    vp, i, f, d, b, sz, ll = (ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_bool,
                              ctypes.c_size_t, ctypes.c_longlong)
    P = ctypes.POINTER
    protos = {
        "aa_py_filterbank_metadata": ([d, d, i, i, d, d, i, d], vp),
        "aa_py_filterbank_metadata_delete": ([vp], None),
        "aa_py_filterbank_metadata_tstart": ([vp], d),
        "aa_py_ddtr_plan": ([], vp),
        "aa_py_ddtr_plan_delete": ([vp], None),
        "aa_py_ddtr_plan_add_dm": ([vp, f, f, f, i, i], b),
        "aa_py_ddtr_plan_range": ([vp], sz),
        "aa_py_ddtr_plan_set_power": ([vp, f], b),
        "aa_py_ddtr_plan_power": ([vp], f),
        "aa_py_ddtr_plan_set_enable_msd_baseline": ([vp, b], b),
        "aa_py_ddtr_plan_enable_msd_baseline_noise": ([vp], b),
        "aa_py_ddtr_plan_bind_bandpass_normalization": ([vp, PFLOAT, i], b),
        "aa_py_pipeline_api": ([aa_py_pipeline_components, aa_py_pipeline_component_options,
                                filterbank_metadata_struct, P(ctypes.c_ushort), i], vp),
        "aa_py_pipeline_api_delete": ([vp], None),
        "aa_py_pipeline_api_bind_ddtr_plan": ([vp, vp], b),
        "aa_py_pipeline_api_ddtr_strategy": ([vp], vp),
        "aa_py_ddtr_strategy_delete": ([vp], None),
        "aa_py_get_ddtr_nRanges": ([vp], sz),
        "aa_py_get_ndms_array": ([vp], P(i)),
        "aa_py_get_t_proc": ([vp, i, i], i),
        "aa_py_dm_low": ([vp, i], i),
        "aa_py_total_computed_samples": ([vp], i),
        "aa_py_pipeline_api_bind_analysis_plan": ([vp, vp], b),
        "aa_py_pipeline_api_bind_periodicity_plan": ([vp, f, b, f, i, i], b),
        "aa_py_pipeline_api_bind_fdas_plan": ([vp, f, f, b], b),
        "aa_py_pipeline_api_run": ([vp, P(i)], b),
        "aa_py_buffer": ([vp], PPPFLOAT),
        "aa_py_current_range": ([vp], i),
        "aa_py_current_time_chunk": ([vp], i),
        "aa_py_current_inc": ([vp], ctypes.c_long),
        "aa_py_cleanup": ([vp], b),
        "aa_b200_strategy": ([P(aa_b200_dm), i, f, i, i, d, d, d, i, sz, i, i, P(f), P(i), P(aa_b200_dm),
                              P(i), P(i), P(i), P(i)], i),
        "aa_b200_select_kernel": ([i, f, f, f, i], i),
        "aa_b200_corner_turn": ([vp, vp, i, i, ll, ll, vp], i),
        "aa_b200_bin_gpu": ([vp, vp, i, i, ll, vp], i),
        "aa_b200_dedisperse": ([i, i, P(i), P(f), vp, ll, sz, vp, ll, i, P(f), P(f), P(f), P(i), i, i, vp], i),
        "aa_b200_dedisperse_noalloc": ([i, i, P(i), P(f), vp, ll, sz, vp, ll, i, P(f), P(f), P(f), P(i), i, i, vp],
                                       i),
        "aa_b200_noalloc_last_error": ([], ctypes.c_char_p),
        "aa_b200_last_error": ([], ctypes.c_char_p),
        "aa_b200_kernel_launches": ([], ll),
        "aa_b200_version": ([], ctypes.c_char_p),
        "aa_b200_pipeline_set_options": ([vp, i, i, i, sz, i, i], b),
        "aa_b200_pipeline_create": ([filterbank_metadata_struct, vp, i, i, i, vp, i], vp),
        "aa_b200_pipeline_set_kernel_variant": ([vp, i], b),
        "aa_b200_pipeline_set_autotune": ([vp, i], b),
        "aa_b200_pipeline_set_packed_input": ([vp, vp], b),
        "aa_b200_selftest_bounded_wait": ([i, P(i)], i),
        "aa_b200_debug_fail_after": ([ll], None),
        "aa_b200_debug_fail_countdown": ([], ll),
        "aa_b200_smem_load_rate": ([i, vp, P(d), P(f)], i),
        "aa_b200_binary_version": ([P(i)], i),
        "aa_b200_pipeline_set_export_base": ([vp, ctypes.c_char_p], b),
        "aa_b200_export_dd_data": ([i, PPPFLOAT, sz, P(i), P(i), ctypes.c_char_p, P(i), i], i),
        "aa_b200_sd_per_file_from_file_size": ([sz, sz, sz], sz),
        "aa_py_sigproc_input": ([ctypes.c_char_p], vp),
        "aa_py_sigproc_input_del": ([vp], None),
        "aa_py_sigproc_input_read_metadata": ([vp], filterbank_metadata_struct),
        "aa_py_sigproc_input_read_signal": ([vp], b),
        "aa_py_sigproc_input_input_buffer": ([vp], P(ctypes.c_ushort)),
        "aa_b200_sigproc_read_packed": ([vp], b),
        "aa_b200_sigproc_packed_buffer": ([vp], vp),
        "aa_b200_sigproc_packed_bytes": ([vp], ll),
        "aa_b200_sigproc_header": ([vp, P(sigproc_header_struct)], b),
        "aa_b200_sigproc_last_error": ([vp], ctypes.c_char_p),
        "aa_b200_pipeline_run_all": ([vp], b),
        "aa_b200_pipeline_setup": ([vp], b),
        "aa_b200_pipeline_rewind": ([vp], b),
        "aa_b200_pipeline_synchronize": ([vp], b),
        "aa_b200_pipeline_device_output": ([vp, i], vp),
        "aa_b200_pipeline_range_info": ([vp, i, P(i), P(i), P(i), P(i)], i),
        "aa_b200_pipeline_kernel_launches": ([vp], ll),
        "aa_b200_pipeline_stage_depth": ([vp, i], i),
        "aa_b200_tuned_ranges": ([i], ll),
        "aa_b200_tuned_ranges_save": ([ctypes.c_char_p], ll),
        "aa_b200_tuned_ranges_load": ([ctypes.c_char_p], ll),
        "aa_b200_tuned_ranges_last_error": ([], ctypes.c_char_p),
        "aa_b200_tuned_ranges_used": ([], ll),
        "aa_b200_pipeline_range_kernel": ([vp, i, P(i), P(i), P(i), P(i)], i),
        "aa_b200_pipeline_last_error": ([vp], ctypes.c_char_p),
        "aa_b200_pipeline_num_tchunks": ([vp], i),
        "aa_b200_pipeline_maxshift": ([vp], i),
        "aa_b200_pipeline_time_kernels": ([vp, i], b),
        "aa_b200_pipeline_kernel_time": ([vp, i, P(d), P(ll)], i),
        "aa_b200_pipeline_reset_kernel_times": ([vp], b),
        "aa_b200_batch_create": ([i, i, sz, i, i, i, vp], vp),
        "aa_b200_batch_add_beam": ([vp, filterbank_metadata_struct, vp, vp], i),
        "aa_b200_batch_setup": ([vp], b),
        "aa_b200_batch_run": ([vp], b),
        "aa_b200_batch_synchronize": ([vp], b),
        "aa_b200_batch_device_output": ([vp, i, i], vp),
        "aa_b200_batch_range_shape": ([vp, i, i, P(i), P(ll), P(i)], i),
        "aa_b200_batch_info": ([vp, P(ll), P(i), P(i), P(i), P(sz), P(sz), P(ll)], i),
        "aa_b200_batch_set_kernel_choice": ([vp, i], b),
        "aa_b200_batch_sub_jobs": ([vp], i),
        "aa_b200_batch_last_ms": ([vp, i], d),
        "aa_b200_batch_estimate_bytes": ([filterbank_metadata_struct, vp, sz, P(sz)], i),
        "aa_b200_batch_last_error": ([vp], ctypes.c_char_p),
        "aa_b200_batch_delete": ([vp], None),
        "aa_b200_frac_dedisperse_fwd": ([vp, vp, vp, vp, i, i, i, vp, vp], i),
        "aa_b200_frac_dedisperse_adj": ([vp, vp, vp, vp, vp, i, i, i, vp, vp, vp, vp], i),
        "aa_b200_boxcar_snr_fwd": ([vp, i, i, P(i), i, vp, vp, vp, vp], i),
        "aa_b200_boxcar_snr_adj": ([vp, i, i, P(i), i, vp, vp, vp], i),
        "aa_b200_frac_last_error": ([], ctypes.c_char_p),
        "aa_b200_sps_row_stats": ([vp, i, ll, ll, vp, vp, vp], i),
        "aa_b200_sps_block_peaks": ([vp, i, ll, ll, vp, vp, P(i), i, vp, vp, vp, vp], i),
        "aa_b200_sps_block_samples": ([], i),
        "aa_py_analysis_plan": ([vp, f, f, f, i, b], vp),
        "aa_analysis_plan_delete": ([vp], None),
        "aa_py_analysis_plan_sigma_cutoff": ([vp], f),
        "aa_py_analysis_plan_sigma_constant": ([vp], f),
        "aa_py_analysis_plan_max_boxcar_width_in_sec": ([vp], f),
        "aa_py_analysis_plan_enable_msd_baseline_noise": ([vp], b),
        "aa_py_spd_nCandidates": ([vp], sz),
        "aa_py_pipeline_api_analysis_strategy": ([vp], vp),
        "aa_py_get_psr_nCandidates": ([vp], P(f)),
        "aa_py_get_psr_interbin_nCandidates": ([vp], P(f)),
        "aa_py_write_to_disk_psr_candidates": ([vp, ctypes.c_char_p], None),
        "aa_b200_pipeline_bind_periodicity_plan": ([vp, f, i, f, i, i, i, i, i, i], b),
        "aa_b200_pipeline_set_periodicity_memory": ([vp, ctypes.c_size_t], b),
        "aa_b200_pipeline_set_device_output": ([vp, i], b),
        "aa_b200_pipeline_psr_count": ([vp, i], ctypes.c_size_t),
        "aa_b200_pipeline_write_psr_interbin_candidates": ([vp, ctypes.c_char_p], b),
        "aa_b200_pipeline_psr_info": ([vp, P(ctypes.c_size_t), P(ctypes.c_size_t), P(i), P(d)], i),
        "aa_py_h_dm": ([vp], P(ctypes.c_uint)),
        "aa_py_h_ts": ([vp], P(ctypes.c_uint)),
        "aa_py_h_snr": ([vp], P(f)),
        "aa_py_h_width": ([vp], P(ctypes.c_uint)),
        "aa_b200_pipeline_set_candidate_output": ([vp, i, ctypes.c_char_p], b),
        "aa_b200_pipeline_set_analysis_batch": ([vp, ll], b),
        "aa_b200_psr_power_interbin": ([vp, vp, vp, i, i, vp], i),
        "aa_b200_psr_harmonic_sum_simple": ([vp, vp, vp, vp, i, i, i, vp], i),
        "aa_b200_psr_kernel_launches": ([], ll),
        "aa_b200_psr_peak_find": ([vp, vp, vp, i, i, f, i, vp, vp, i, i, i, i, vp], i),
        "aa_b200_psr_threshold": ([vp, vp, vp, i, i, f, i, vp, vp, i, i, i, i, vp], i),
        "aa_b200_psr_harmonic_sum": ([i, vp, vp, vp, vp, i, i, i, i, vp], i),
        "aa_b200_psr_last_error": ([], ctypes.c_char_p),
        "aa_b200_psr_whitening": ([vp, ctypes.c_size_t, i, vp], i),
        "aa_b200_psr_segment_sizes": ([ctypes.c_size_t, vp, i], i),
        "aa_b200_psr_segment_medians": ([vp, ctypes.c_size_t, i, vp, i, vp, vp], i),
        "aa_b200_psr_candidates_process": ([vp, ctypes.c_size_t, vp, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_size_t, f, i], i),
        "aa_b200_psr_candidates_create": ([], vp),
        "aa_b200_psr_candidates_destroy": ([vp], None),
        "aa_b200_psr_candidates_add": ([vp, vp, ctypes.c_size_t, i, i, vp, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_size_t, f, i], i),
        "aa_b200_psr_candidates_count": ([vp], ctypes.c_size_t),
        "aa_b200_psr_candidates_copy": ([vp, vp], i),
        "aa_b200_psr_candidates_export": ([vp, ctypes.c_char_p], i),
        "aa_b200_psr_candidates_last_error": ([], ctypes.c_char_p),
        "aa_b200_spd_create": ([ll, ll], vp),
        "aa_b200_spd_destroy": ([vp], None),
        "aa_b200_spd_last_error": ([vp], ctypes.c_char_p),
        "aa_b200_spd_clear": ([vp, vp], i),
        "aa_b200_spd_run": ([vp, vp, i, i, f, i, f, f, f, i, i, vp, sz, vp, vp, vp, vp, P(sz)], i),
        "aa_b200_spd_profile": ([vp, vp, i, vp, P(i), P(i), P(i), P(i)], i),
        "aa_b200_spd_keep_planes": ([vp, i], i),
        "aa_b200_spd_planes": ([vp, vp, vp, ll], ll),
        "aa_b200_spd_kernel_launches": ([], ll),
        "aa_b200_spd_plan": ([i, f, i, f, vp, i, P(i), P(i), P(i), vp, i, P(i)], i),
        "aa_b200_spd_msd_profile": ([vp, vp, i, i, P(i), i, i, f, i, vp, vp], i),
        "aa_b200_spd_time_kernels": ([vp, i], i),
        "aa_b200_spd_first_plane": ([vp, vp, vp, vp, vp, vp, i, i, i, vp], i),
        "aa_b200_spd_family_time": ([vp, i, P(d), P(ll)], i),
        "aa_b200_spd_write_candidates": ([ctypes.c_char_p, i, f, f, f, f, f, i, vp, vp, vp, vp, sz], i),
    }
    for name, (args, res) in protos.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def declared_symbols() -> list:
    """Every function name include/aa_b200.h declares."""
    import re
    hdr = os.path.join(os.path.dirname(PKG_ROOT), "include", "aa_b200.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(aa_(?:py|b200)_\w+)\s*\(", text)))


def smem_load_rate(iters: int = 4096, stream=None) -> dict:
    """Measured 32-bit shared-memory loads per second of this GPU (see
    aa_b200_smem_load_rate) and the adds/s bound it sets for the
    channel-quad kernel (four channel adds per load)."""
    rate, ms = ctypes.c_double(), ctypes.c_float()
    if lib().aa_b200_smem_load_rate(iters, stream, ctypes.byref(rate), ctypes.byref(ms)) != 0:
        raise RuntimeError("shared-memory load-rate measurement failed")
    return {"loads_per_s": rate.value, "adds_per_s": 4.0 * rate.value, "ms": ms.value, "iters": iters}


def last_error() -> str:
    return lib().aa_b200_last_error().decode()


# ---------------------------------------------------------------------------
# Reference-facing classes (cmake/py_astro_accelerate.py.in)
# ---------------------------------------------------------------------------
class aa_py_filterbank_metadata:
    def __init__(self, tstart: float, tsamp: float, nbits: int, nsamples: int, fch1: float, foff: float,
                 nchans: int, src_raj: float = 0.0):
        self.m_tstart, self.m_tsamp, self.m_nbits, self.m_nsamples = tstart, tsamp, nbits, nsamples
        self.m_fch1, self.m_foff, self.m_nchans, self.m_src_raj = fch1, foff, nchans, src_raj
        self.m_obj = lib().aa_py_filterbank_metadata(tstart, tsamp, nbits, nsamples, fch1, foff, nchans, src_raj)

    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc_value, traceback):
        lib().aa_py_filterbank_metadata_delete(self.m_obj)

    def pointer(self):
        return self.m_obj

    def tstart(self):
        return lib().aa_py_filterbank_metadata_tstart(self.m_obj)

    def struct(self) -> filterbank_metadata_struct:
        return filterbank_metadata_struct(self.m_tstart, self.m_tsamp, self.m_fch1, self.m_foff, self.m_nbits,
                                          self.m_nsamples, self.m_nchans, self.m_src_raj)


class aa_py_dm:
    def __init__(self, low: float, high: float, step: float, inBin: int, outBin: int):
        self.m_low, self.m_high, self.m_step, self.m_inBin, self.m_outBin = low, high, step, inBin, outBin

    def low(self):
        return self.m_low

    def high(self):
        return self.m_high

    def step(self):
        return self.m_step

    def inBin(self):
        return self.m_inBin

    def outBin(self):
        return self.m_outBin


class aa_py_ddtr_plan:
    def __init__(self, dm):
        self.m_obj = lib().aa_py_ddtr_plan()
        self.m_dm = list(dm)
        for r in self.m_dm:
            lib().aa_py_ddtr_plan_add_dm(self.m_obj, r.low(), r.high(), r.step(), r.inBin(), r.outBin())

    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc_value, traceback):
        self.delete()

    def delete(self):
        if self.m_obj:
            lib().aa_py_ddtr_plan_delete(self.m_obj)
            self.m_obj = None

    def pointer(self):
        return self.m_obj

    def set_power(self, power: float):
        return lib().aa_py_ddtr_plan_set_power(self.m_obj, power)

    def power(self):
        return lib().aa_py_ddtr_plan_power(self.m_obj)

    def set_enable_msd_baseline_noise(self, flag: bool):
        return lib().aa_py_ddtr_plan_set_enable_msd_baseline(self.m_obj, flag)

    def enable_msd_baseline_noise(self):
        return lib().aa_py_ddtr_plan_enable_msd_baseline_noise(self.m_obj)

    def bind_bandpass_normalization(self, data, data_size: int):
        arr = np.ascontiguousarray(data, dtype=np.float32)
        return lib().aa_py_ddtr_plan_bind_bandpass_normalization(self.m_obj, arr.ctypes.data_as(PFLOAT), data_size)

    def range(self):
        return lib().aa_py_ddtr_plan_range(self.m_obj)


class aa_py_analysis_plan:
    """The single-pulse detection settings (cmake/py_astro_accelerate.py.in
    aa_py_analysis_plan): candidate_algorithm 0 peak finding, 1 thresholding,
    2 peak filtering."""

    def __init__(self, sigma_cutoff: float, sigma_constant: float, max_boxcar_width_in_sec: float,
                 candidate_algorithm: int, enable_msd_baseline_noise: bool):
        self.m_sigma_cutoff = sigma_cutoff
        self.m_sigma_constant = sigma_constant
        self.m_max_boxcar_width_in_sec = max_boxcar_width_in_sec
        self.m_candidate_algorithm = candidate_algorithm
        self.m_enable_msd_baseline_noise = enable_msd_baseline_noise

    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc_value, traceback):
        pass

    def sigma_cutoff(self):
        return self.m_sigma_cutoff

    def sigma_constant(self):
        return self.m_sigma_constant

    def max_boxcar_width_in_sec(self):
        return self.m_max_boxcar_width_in_sec

    def candidate_algorithm(self):
        return self.m_candidate_algorithm

    def enable_msd_baseline_noise(self):
        return self.m_enable_msd_baseline_noise


class aa_py_periodicity_plan:
    """cmake/py_astro_accelerate.py.in:298-330: the periodicity settings the
    reference's wrapper passes to aa_py_pipeline_api_bind_periodicity_plan
    (sigma_constant is the outlier-rejection sigma, enable_msd_baseline_noise
    switches outlier rejection on; export_powers is kept and unused, as
    there)."""

    def __init__(self, sigma_cutoff: float, sigma_constant: float, nHarmonics: int, export_powers: int,
                 candidate_algorithm: int, enable_msd_baseline_noise: bool):
        self.m_sigma_cutoff = sigma_cutoff
        self.m_sigma_constant = sigma_constant
        self.m_nHarmonics = nHarmonics
        self.m_export_powers = export_powers
        self.m_candidate_algorithm = candidate_algorithm
        self.m_enable_msd_baseline_noise = enable_msd_baseline_noise

    def sigma_cutoff(self):
        return self.m_sigma_cutoff

    def sigma_constant(self):
        return self.m_sigma_constant

    def nHarmonics(self):
        return self.m_nHarmonics

    def export_powers(self):
        return self.m_export_powers

    def candidate_algorithm(self):
        return self.m_candidate_algorithm

    def candidate_selection_algorithm(self):
        return int(self.m_candidate_algorithm)

    def enable_msd_baseline_noise(self):
        return self.m_enable_msd_baseline_noise


class aa_py_pipeline:
    """aa_pipeline_api<unsigned short> through the C ABI."""

    def __init__(self, pipeline: aa_py_pipeline_components, pipeline_options: aa_py_pipeline_component_options,
                 metadata: filterbank_metadata_struct, input_data, card_number: int):
        if isinstance(input_data, np.ndarray):
            self._input_keepalive = input_data
            input_data = input_data.ctypes.data_as(ctypes.POINTER(ctypes.c_ushort))
        self.m_obj = lib().aa_py_pipeline_api(pipeline, pipeline_options, metadata, input_data, card_number)
        self.m_status_code_c_int = ctypes.c_int(0)

    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc_value, traceback):
        self.delete()

    def delete(self):
        if self.m_obj:
            lib().aa_py_pipeline_api_delete(self.m_obj)
            self.m_obj = None

    def bind_ddtr_plan(self, plan: aa_py_ddtr_plan):
        return lib().aa_py_pipeline_api_bind_ddtr_plan(self.m_obj, plan.pointer())

    def ddtr_strategy(self):
        return lib().aa_py_pipeline_api_ddtr_strategy(self.m_obj)

    def ddtr_range(self):
        return lib().aa_py_get_ddtr_nRanges(self.m_obj)

    def ddtr_ndms(self):
        return lib().aa_py_get_ndms_array(self.m_obj)

    def bind_analysis_plan(self, plan: "aa_py_analysis_plan"):
        """The analysis plan over this pipeline's DDTR strategy (bind the DDTR
        plan first), as the reference's wrapper does."""
        strat = lib().aa_py_pipeline_api_ddtr_strategy(self.m_obj)
        ptr = lib().aa_py_analysis_plan(strat, plan.sigma_cutoff(), plan.sigma_constant(),
                                        plan.max_boxcar_width_in_sec(), int(plan.candidate_algorithm()),
                                        bool(plan.enable_msd_baseline_noise()))
        if strat:
            lib().aa_py_ddtr_strategy_delete(strat)
        self.m_analysis_plan_ptr = ptr
        return bool(lib().aa_py_pipeline_api_bind_analysis_plan(self.m_obj, ptr))

    def get_candidates(self):
        """After a run() step with status 1 (has_more): nCandidates, dm,
        time_sample, snr, width (ctypes arrays), current_range,
        current_tchunk, current_inc -- the position after the step, as the
        reference's wrapper returns it."""
        if self.m_status_code_c_int.value == 1:
            n = lib().aa_py_spd_nCandidates(self.m_obj)
            return (n, lib().aa_py_h_dm(self.m_obj), lib().aa_py_h_ts(self.m_obj), lib().aa_py_h_snr(self.m_obj),
                    lib().aa_py_h_width(self.m_obj), lib().aa_py_current_range(self.m_obj),
                    lib().aa_py_current_time_chunk(self.m_obj), lib().aa_py_current_inc(self.m_obj))
        return None, [], [], [], [], None, None, None

    def candidates(self) -> dict:
        """The last step's candidates as numpy arrays (dm, ts, snr, bw)."""
        n = lib().aa_py_spd_nCandidates(self.m_obj)
        out = {}
        for key, fn, dt in (("dm", lib().aa_py_h_dm, np.uint32), ("ts", lib().aa_py_h_ts, np.uint32),
                            ("snr", lib().aa_py_h_snr, np.float32), ("bw", lib().aa_py_h_width, np.uint32)):
            ptr = fn(self.m_obj)
            out[key] = np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, dt)
        return out

    def set_candidate_output(self, write_files: bool = True, directory: str | None = None):
        """Whether and where the reference's candidate files are written."""
        return bool(lib().aa_b200_pipeline_set_candidate_output(self.m_obj, int(write_files),
                                                                os.fsencode(directory) if directory else None))

    def set_analysis_batch(self, max_time_samples: int):
        if not lib().aa_b200_pipeline_set_analysis_batch(self.m_obj, int(max_time_samples)):
            raise ValueError(self.last_error())
        return True

    def bind_periodicity_plan(self, plan: "aa_py_periodicity_plan"):
        """cmake/py_astro_accelerate.py.in:476-479: the plan's sigma cutoff,
        outlier rejection (its enable_msd_baseline_noise), outlier sigma (its
        sigma_constant), harmonics and candidate algorithm; the greedy
        harmonic sum with scalloping-loss mitigation."""
        return bool(lib().aa_py_pipeline_api_bind_periodicity_plan(
            self.m_obj, plan.sigma_cutoff(), bool(plan.enable_msd_baseline_noise()), plan.sigma_constant(),
            int(plan.nHarmonics()), int(plan.candidate_selection_algorithm())))

    def bind_periodicity_plan_full(self, sigma_cutoff=10.0, enable_outlier_rejection=True,
                                   sigma_outlier_rejection_threshold=3.0, nHarmonics=32, harmonic_sum_algorithm=1,
                                   candidate_selection_algorithm=0, enable_scalloping_loss_mitigation=True,
                                   enable_interbinning=True, enable_spectrum_whitening=True):
        """aa_periodicity_plan's ten-argument constructor
        (include/aa_periodicity_plan.hpp:62-89): any harmonic sum algorithm
        (0 simple, 1 greedy, 2 PRESTO plus, 3 PRESTO)."""
        return bool(lib().aa_b200_pipeline_bind_periodicity_plan(
            self.m_obj, float(sigma_cutoff), int(bool(enable_outlier_rejection)),
            float(sigma_outlier_rejection_threshold), int(nHarmonics), int(harmonic_sum_algorithm),
            int(candidate_selection_algorithm), int(bool(enable_scalloping_loss_mitigation)),
            int(bool(enable_interbinning)), int(bool(enable_spectrum_whitening))))

    def set_device_output(self, on: bool = True):
        """Keep every range's output on the device too (before the DDTR plan
        is bound); the periodicity search then reads the device rows."""
        if not lib().aa_b200_pipeline_set_device_output(self.m_obj, int(bool(on))):
            raise ValueError(self.last_error())

    def set_periodicity_memory(self, nbytes: int):
        """Bytes the periodicity strategy plans for (default: the device's
        free memory when the plan is bound, as the reference takes it)."""
        if not lib().aa_b200_pipeline_set_periodicity_memory(self.m_obj, int(nbytes)):
            raise ValueError(self.last_error())

    def get_psr_candidates(self, interbin: bool = False) -> np.ndarray:
        """The periodicity candidates [n][4] (DM, frequency, S/N, harmonics)
        of the power (or interbin) spectra, as aa_py_get_psr_nCandidates /
        aa_py_get_psr_interbin_nCandidates give them."""
        n = lib().aa_b200_pipeline_psr_count(self.m_obj, int(bool(interbin)))
        fn = lib().aa_py_get_psr_interbin_nCandidates if interbin else lib().aa_py_get_psr_nCandidates
        ptr = fn(self.m_obj)
        if not ptr:
            raise RuntimeError(self.last_error())
        return np.ctypeslib.as_array(ptr, shape=(4 * n + 4,))[:4 * n].reshape(n, 4).copy()

    def write_psr_candidates(self, filename: str, interbin: bool = False):
        if interbin:
            if not lib().aa_b200_pipeline_write_psr_interbin_candidates(self.m_obj, filename.encode()):
                raise RuntimeError(self.last_error())
        else:
            lib().aa_py_write_to_disk_psr_candidates(self.m_obj, filename.encode())

    def psr_info(self) -> dict:
        fl, dpb, nb, ms = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_int(), ctypes.c_double()
        if lib().aa_b200_pipeline_psr_info(self.m_obj, ctypes.byref(fl), ctypes.byref(dpb), ctypes.byref(nb),
                                           ctypes.byref(ms)):
            raise RuntimeError("no periodicity plan bound")
        return {"fft_length": fl.value, "dms_per_batch": dpb.value, "batches": nb.value, "compute_ms": ms.value}

    def bind_fdas_plan(self, plan):
        return lib().aa_py_pipeline_api_bind_fdas_plan(self.m_obj, 0.0, 0.0, False)

    def run(self):
        return bool(lib().aa_py_pipeline_api_run(self.m_obj, ctypes.byref(self.m_status_code_c_int)))

    def status_code(self):
        return self.m_status_code_c_int.value

    def get_buffer(self):
        return lib().aa_py_total_computed_samples(self.m_obj), lib().aa_py_buffer(self.m_obj)

    def dm_low(self, pos: int):
        return lib().aa_py_dm_low(self.m_obj, pos)

    def t_processed(self, i: int, j: int):
        return lib().aa_py_get_t_proc(self.m_obj, i, j)

    def cleanUp(self):
        return bool(lib().aa_py_cleanup(self.m_obj))

    # ---- extensions of this library ----
    def set_options(self, stride_mode=STRIDE_REFERENCE, fma_mode=7, failsafe=0, free_memory=0, tile_words=0,
                    group_dms=0):
        ok = lib().aa_b200_pipeline_set_options(self.m_obj, stride_mode, fma_mode, failsafe, free_memory,
                                                 tile_words, group_dms)
        if not ok:
            raise ValueError(self.last_error())
        return ok

    def set_packed_input(self, packed):
        """Read the SIGPROC data section as stored instead of the unsigned-short
        input (before bind): a uint8 array [nsamples][nchans*nbits/8] (a 16-bit
        array for nbits 16 and 32), or a pointer (int)."""
        if isinstance(packed, np.ndarray):
            if not packed.flags["C_CONTIGUOUS"]:
                raise ValueError("the packed input must be C-contiguous")
            self._packed_keepalive = packed
            packed = packed.ctypes.data
        if not lib().aa_b200_pipeline_set_packed_input(self.m_obj, ctypes.c_void_p(packed)):
            raise ValueError(self.last_error())
        return True

    def set_export_base(self, base: str):
        """Base name of the output_dmt files (default "DD_data" in the working directory)."""
        if not lib().aa_b200_pipeline_set_export_base(self.m_obj, os.fsencode(base)):
            raise ValueError(self.last_error())
        return True

    def set_kernel_variant(self, variant: int):
        """Kernel family per range (before bind): 0 auto (timed per range), 1
        generic kernels, 2 channel-quad / fp32, 3 subband / fp32, 4
        warp-specialised channel-quad / fp32, 5 split-phase channel-quad /
        fp32, 6 channel-quad with reuse by offset pattern / fp32, 7
        channel-quad on 256-sample tiles, two CTAs per SM / fp32."""
        if not lib().aa_b200_pipeline_set_kernel_variant(self.m_obj, variant):
            raise ValueError(self.last_error())
        return True

    def set_autotune(self, enable: bool):
        """Time the staged kernels per range at set-up (default on)."""
        if not lib().aa_b200_pipeline_set_autotune(self.m_obj, int(bool(enable))):
            raise ValueError(self.last_error())
        return True

    def run_all(self):
        return bool(lib().aa_b200_pipeline_run_all(self.m_obj))

    def setup(self):
        """Device buffers, tables and the autotuner now rather than at the
        first run."""
        return bool(lib().aa_b200_pipeline_setup(self.m_obj))

    def rewind(self):
        return bool(lib().aa_b200_pipeline_rewind(self.m_obj))

    def synchronize(self):
        return bool(lib().aa_b200_pipeline_synchronize(self.m_obj))

    def last_error(self) -> str:
        return lib().aa_b200_pipeline_last_error(self.m_obj).decode()

    def kernel_launches(self) -> int:
        return lib().aa_b200_pipeline_kernel_launches(self.m_obj)

    def num_tchunks(self) -> int:
        return lib().aa_b200_pipeline_num_tchunks(self.m_obj)

    def maxshift(self) -> int:
        return lib().aa_b200_pipeline_maxshift(self.m_obj)

    def range_info(self, r: int) -> dict:
        k, g, s, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        if lib().aa_b200_pipeline_range_info(self.m_obj, r, ctypes.byref(k), ctypes.byref(g), ctypes.byref(s),
                                              ctypes.byref(t)):
            raise RuntimeError(self.last_error())
        return {"kind": KIND_NAMES[k.value & 0xFF], "kernel": ("quad" if k.value & 0x100 else "f32" if k.value & 0x200 else
                           "gather" if k.value & 0x400 else "sub" if k.value & 0x800 else "quadws" if k.value & 0x1000
                           else "quadsp" if k.value & 0x2000 else "phase"),
                "stage_depth": lib().aa_b200_pipeline_stage_depth(self.m_obj, r),
                "group_dms": g.value, "span": s.value, "tile_words": t.value, **self.range_kernel(r)}

    def range_kernel(self, r: int) -> dict:
        """The kernel shape range r runs after set-up: channel-quad flavour
        (-1 for other kernels), output tile (DM trials x samples per CTA) and
        DM trials per warp."""
        f, d, t, w = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        if lib().aa_b200_pipeline_range_kernel(self.m_obj, r, ctypes.byref(f), ctypes.byref(d), ctypes.byref(t),
                                               ctypes.byref(w)):
            raise RuntimeError(self.last_error())
        return {"flavour": f.value, "tile": [d.value, t.value], "dms_per_warp": w.value}

    def time_kernels(self, on: bool = True):
        return bool(lib().aa_b200_pipeline_time_kernels(self.m_obj, int(on)))

    def kernel_time(self, family: int = 0):
        """(ms, launches) of a kernel family: 0 dedispersion, 1 corner turn, 2 binning."""
        ms, n = ctypes.c_double(), ctypes.c_longlong()
        if lib().aa_b200_pipeline_kernel_time(self.m_obj, family, ctypes.byref(ms), ctypes.byref(n)):
            raise RuntimeError(self.last_error())
        return ms.value, n.value

    def reset_kernel_times(self):
        return bool(lib().aa_b200_pipeline_reset_kernel_times(self.m_obj))

    def device_output(self, r: int) -> int:
        return lib().aa_b200_pipeline_device_output(self.m_obj, r) or 0

    def output_arrays(self):
        """The host output rows as numpy arrays [range] -> (ndms, total_samps).

        Rows of one range are contiguous in this library's pinned output block,
        so each range is one zero-copy view."""
        nr = self.ddtr_range()
        ndms = self.ddtr_ndms()
        buf = lib().aa_py_buffer(self.m_obj)
        nt = self.num_tchunks()
        out = []
        for r in range(nr):
            tot = sum(self.t_processed(r, k) for k in range(nt))
            n = ndms[r]
            base = ctypes.cast(buf[r][0], ctypes.c_void_p).value
            arr = np.ctypeslib.as_array((ctypes.c_float * (n * tot)).from_address(base)).reshape(n, tot)
            out.append(arr)
        return out


class aa_py_sigproc_input:
    """SIGPROC filterbank reader (the reference's aa_py_sigproc_input,
    cmake/py_astro_accelerate.py.in:71-101): read_metadata, read_signal and
    input_buffer as there, plus numpy views and the packed read."""

    def __init__(self, path: str):
        self.m_obj = lib().aa_py_sigproc_input(os.fsencode(path))
        self._meta = None

    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc_value, traceback):
        self.delete()

    def delete(self):
        if self.m_obj:
            lib().aa_py_sigproc_input_del(self.m_obj)
            self.m_obj = None

    def read_metadata(self) -> filterbank_metadata_struct:
        self._meta = lib().aa_py_sigproc_input_read_metadata(self.m_obj)
        return self._meta

    def read_signal(self) -> bool:
        return bool(lib().aa_py_sigproc_input_read_signal(self.m_obj))

    def input_buffer(self):
        """ctypes pointer to [nsamples][nchans] unsigned short (as the reference)."""
        return lib().aa_py_sigproc_input_input_buffer(self.m_obj)

    def input_array(self) -> np.ndarray:
        """input_buffer as a [nsamples][nchans] uint16 view (valid while this object lives)."""
        m = self._meta
        p = self.input_buffer()
        if m is None or not p:
            raise RuntimeError("read_metadata and read_signal first: " + self.last_error())
        return np.ctypeslib.as_array(p, shape=(m.m_nsamples, m.m_nchans))

    def read_packed(self) -> bool:
        return bool(lib().aa_b200_sigproc_read_packed(self.m_obj))

    def packed_array(self) -> np.ndarray:
        """The data section as stored, [nsamples][record bytes] uint8 (16-bit
        [nsamples][nchans] for nbits 16 and 32)."""
        m = self._meta
        n = lib().aa_b200_sigproc_packed_bytes(self.m_obj)
        p = lib().aa_b200_sigproc_packed_buffer(self.m_obj)
        if m is None or not p:
            raise RuntimeError("read_metadata and read_packed first: " + self.last_error())
        raw = np.ctypeslib.as_array((ctypes.c_uint8 * n).from_address(p))
        if m.m_nbits >= 16:
            return raw.view(np.uint16).reshape(m.m_nsamples, m.m_nchans)
        return raw.reshape(m.m_nsamples, -1) if m.m_nsamples else raw.reshape(0, 0)

    def header(self) -> dict:
        h = sigproc_header_struct()
        if not lib().aa_b200_sigproc_header(self.m_obj, ctypes.byref(h)):
            raise RuntimeError(self.last_error())
        return {k: getattr(h, k) for k, _ in h._fields_}

    def last_error(self) -> str:
        e = lib().aa_b200_sigproc_last_error(self.m_obj)
        return e.decode() if e else ""


def create_pipeline(metadata: filterbank_metadata_struct, input_ptr: int, device_input: bool,
                    device_output: bool, copy_to_host: bool, stream: int = 0, card_number: int = 0):
    """A pipeline over device-resident input and/or output (this library's extension)."""
    p = aa_py_pipeline.__new__(aa_py_pipeline)
    p.m_obj = lib().aa_b200_pipeline_create(metadata, ctypes.c_void_p(input_ptr), int(device_input),
                                            int(device_output), int(copy_to_host), ctypes.c_void_p(stream),
                                            card_number)
    p.m_status_code_c_int = ctypes.c_int(0)
    return p


# ---------------------------------------------------------------------------
# Seam (stateless)
# ---------------------------------------------------------------------------
def strategy(plan, nchans, nsamp, fch1, foff, tsamp, nbits, free_memory=180 * 2**30, power=2.0,
             enable_analysis=False, max_chunks=4096):
    """The reference strategy computed by this library's planner (host only)."""
    L = lib()
    nr = len(plan)
    parr = (aa_b200_dm * nr)(*[aa_b200_dm(*p) for p in plan])
    dmshifts = np.zeros(nchans, np.float32)
    ndms = (ctypes.c_int * nr)()
    sdm = (aa_b200_dm * nr)()
    ms, mx, nt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    tp = np.zeros(nr * max_chunks, np.int32)
    rc = L.aa_b200_strategy(parr, nr, power, nchans, nsamp, fch1, foff, tsamp, nbits, free_memory,
                            int(enable_analysis), max_chunks, dmshifts.ctypes.data_as(PFLOAT), ndms, sdm,
                            ctypes.byref(ms), ctypes.byref(mx), ctypes.byref(nt),
                            tp.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    if rc != 0:
        raise ValueError(f"strategy refused the plan (code {rc})")
    return {
        "dmshifts": dmshifts,
        "ndms": [int(ndms[r]) for r in range(nr)],
        "dm": [(sdm[r].low, sdm[r].high, sdm[r].step, sdm[r].inBin, sdm[r].outBin) for r in range(nr)],
        "maxshift": ms.value,
        "max_ndms": mx.value,
        "num_tchunks": nt.value,
        "t_processed": [[int(tp[r * max_chunks + k]) for k in range(nt.value)] for r in range(nr)],
    }


def select_kernel(nbits, dm_step, tsamp, dmshift_last, failsafe=0) -> int:
    return lib().aa_b200_select_kernel(nbits, dm_step, tsamp, dmshift_last, failsafe)


def _ptr(x) -> int:
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    return int(x)


def corner_turn(d_in_tc, d_out, nbits, nchans, nsamp, out_stride, stream=0):
    if lib().aa_b200_corner_turn(_ptr(d_in_tc), _ptr(d_out), nbits, nchans, nsamp, out_stride, stream):
        raise RuntimeError(last_error())


def bin_gpu(d_src, d_dst, nbits, nchans, nsamp, stream=0):
    if lib().aa_b200_bin_gpu(_ptr(d_src), _ptr(d_dst), nbits, nchans, nsamp, stream):
        raise RuntimeError(last_error())


def _dedisperse_args(i, t_processed, inBin, dmshifts, d_input, i_nsamp, d_input_elems, d_output, out_pitch, nchans,
                     tsamp, dm_low, dm_step, ndms, nbits, failsafe, stream):
    nr = len(ndms)
    keep = dict(inb=(ctypes.c_int * nr)(*inBin), sh=np.ascontiguousarray(dmshifts, dtype=np.float32),
                ts=ctypes.c_float(tsamp), lo=(ctypes.c_float * nr)(*dm_low), st=(ctypes.c_float * nr)(*dm_step),
                nd=(ctypes.c_int * nr)(*ndms))
    args = (i, t_processed, keep["inb"], keep["sh"].ctypes.data_as(PFLOAT), _ptr(d_input), i_nsamp, d_input_elems,
            _ptr(d_output), out_pitch, nchans, ctypes.byref(keep["ts"]), keep["lo"], keep["st"], keep["nd"], nbits,
            failsafe, stream)
    return args, keep


def dedisperse_noalloc(i, t_processed, inBin, dmshifts, d_input, i_nsamp, d_input_elems, d_output, out_pitch,
                       nchans, tsamp, dm_low, dm_step, ndms, nbits, failsafe=0, stream=0):
    """aa_b200_dedisperse_noalloc: the same work with the library's fixed
    device scratch array instead of allocated scratch."""
    args, keep = _dedisperse_args(i, t_processed, inBin, dmshifts, d_input, i_nsamp, d_input_elems, d_output,
                                  out_pitch, nchans, tsamp, dm_low, dm_step, ndms, nbits, failsafe, stream)
    if lib().aa_b200_dedisperse_noalloc(*args):
        raise RuntimeError(lib().aa_b200_noalloc_last_error().decode())


def dedisperse(i, t_processed, inBin, dmshifts, d_input, i_nsamp, d_input_elems, d_output, out_pitch, nchans,
               tsamp, dm_low, dm_step, ndms, nbits, failsafe=0, stream=0):
    """dedisperse() of src/aa_dedisperse.cpp:5 with explicit stride, size and stream."""
    nr = len(ndms)
    inb = (ctypes.c_int * nr)(*inBin)
    sh = np.ascontiguousarray(dmshifts, dtype=np.float32)
    ts = ctypes.c_float(tsamp)
    lo = (ctypes.c_float * nr)(*dm_low)
    st = (ctypes.c_float * nr)(*dm_step)
    nd = (ctypes.c_int * nr)(*ndms)
    rc = lib().aa_b200_dedisperse(i, t_processed, inb, sh.ctypes.data_as(PFLOAT), _ptr(d_input), i_nsamp,
                                  d_input_elems, _ptr(d_output), out_pitch, nchans, ctypes.byref(ts), lo, st, nd,
                                  nbits, failsafe, stream)
    if rc:
        raise RuntimeError(last_error())


# ---------------------------------------------------------------------------
# Multi-beam batch (one CUDA graph, one persistent dedispersion kernel)
# ---------------------------------------------------------------------------
class _DeviceRows:
    """__cuda_array_interface__ of a float32 device array owned by the library."""

    def __init__(self, ptr: int, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4", "data": (ptr, False),
                                         "version": 2, "strides": None}


class batch:
    """Many beams' DDTR in one graph (aa_b200_batch_*).  Inputs are
    [nsamples][nchans] uint16 device buffers (torch tensors or pointers) that
    must stay alive while the batch runs."""

    def __init__(self, stride_mode: int = STRIDE_REFERENCE, fma_mode: int = 7, free_memory: int = 0,
                 persistent: bool = True, use_graph: bool = True, autotune: bool = True, stream: int = 0):
        self.m_obj = lib().aa_b200_batch_create(stride_mode, fma_mode, free_memory, int(persistent), int(use_graph),
                                                int(autotune), ctypes.c_void_p(stream))
        if not self.m_obj:
            raise RuntimeError(self.last_error())
        self._keep = []

    def last_error(self) -> str:
        m = lib().aa_b200_batch_last_error(getattr(self, "m_obj", None))
        return m.decode() if m else ""

    def add_beam(self, metadata: filterbank_metadata_struct, plan: "aa_py_ddtr_plan", d_input) -> int:
        ptr = d_input if isinstance(d_input, int) else d_input.data_ptr()
        self._keep.append(d_input)
        i = lib().aa_b200_batch_add_beam(self.m_obj, metadata, plan.pointer(), ctypes.c_void_p(ptr))
        if i < 0:
            raise RuntimeError(self.last_error())
        return i

    def _check(self, ok):
        if not ok:
            raise RuntimeError(self.last_error())
        return True

    def set_kernel_choice(self, choice: int):
        """One-byte ranges both bodies can run (before setup): 0 the faster
        on a timed slice, 1 channel-quad, 2 subband."""
        return self._check(lib().aa_b200_batch_set_kernel_choice(self.m_obj, int(choice)))

    def sub_jobs(self) -> int:
        """Persistent jobs the subband body runs (after setup)."""
        return int(lib().aa_b200_batch_sub_jobs(self.m_obj))

    def setup(self):
        return self._check(lib().aa_b200_batch_setup(self.m_obj))

    def run(self):
        return self._check(lib().aa_b200_batch_run(self.m_obj))

    def synchronize(self):
        return self._check(lib().aa_b200_batch_synchronize(self.m_obj))

    def range_shape(self, beam: int, r: int):
        n, t, b = ctypes.c_int(), ctypes.c_longlong(), ctypes.c_int()
        if lib().aa_b200_batch_range_shape(self.m_obj, beam, r, ctypes.byref(n), ctypes.byref(t), ctypes.byref(b)):
            raise RuntimeError(self.last_error())
        return n.value, t.value, b.value

    def output(self, beam: int, r: int):
        """Zero-copy torch view (ndms, total_samps) of one range of one beam."""
        import torch
        ptr = lib().aa_b200_batch_device_output(self.m_obj, beam, r)
        if not ptr:
            raise RuntimeError("no output for this beam/range (is the batch set up?)")
        ndms, tot, _ = self.range_shape(beam, r)
        return torch.as_tensor(_DeviceRows(ptr, (ndms, tot)), device="cuda")

    def info(self) -> dict:
        w, pj, oj, g, sm, lb, lp = (ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int(),
                                    ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_longlong())
        lib().aa_b200_batch_info(self.m_obj, *(ctypes.byref(v) for v in (w, pj, oj, g, sm, lb, lp)))
        return {"work_items": w.value, "persistent_jobs": pj.value, "other_jobs": oj.value, "grid": g.value,
                "smem_bytes": sm.value, "level_bytes": lb.value, "launches_per_run": lp.value}

    def last_ms(self, which: int = 0) -> float:
        return lib().aa_b200_batch_last_ms(self.m_obj, which)

    def delete(self):
        if getattr(self, "m_obj", None):
            lib().aa_b200_batch_delete(self.m_obj)
            self.m_obj = None
            self._keep = []


def batch_estimate_bytes(metadata: filterbank_metadata_struct, plan: "aa_py_ddtr_plan", free_memory: int) -> int:
    n = ctypes.c_size_t()
    if lib().aa_b200_batch_estimate_bytes(metadata, plan.pointer(), free_memory, ctypes.byref(n)):
        raise RuntimeError(lib().aa_b200_batch_last_error(None).decode())
    return n.value


class single_pulse_detection:
    """analysis_GPU (src/aa_device_analysis.cu:130-345) on DM-time planes in
    device memory (aa_b200_spd_*): the reference's MSD profile, boxcar S/N
    planes and candidate lists (peak finding, thresholding or peak
    filtering), bit for bit.

    max_elems bounds nDMs * nT of the planes run; max_time_samples is the
    reference's batch size in elements (0 = one batch for the whole plane).
    run() overwrites the plane, like the reference's search."""

    def __init__(self, max_elems: int, max_time_samples: int = 0):
        self.m_obj = lib().aa_b200_spd_create(int(max_elems), int(max_time_samples))
        if not self.m_obj:
            raise RuntimeError(lib().aa_b200_spd_last_error(None).decode())

    def last_error(self) -> str:
        m = lib().aa_b200_spd_last_error(self.m_obj)
        return m.decode() if m else ""

    def clear(self, stream: int = 0):
        if lib().aa_b200_spd_clear(self.m_obj, ctypes.c_void_p(stream)):
            raise RuntimeError(self.last_error())

    def keep_planes(self, on: bool = True):
        lib().aa_b200_spd_keep_planes(self.m_obj, int(on))

    def run(self, d_plane, ndms: int, nt: int, tsamp: float, inBin: int, sigma_cutoff: float, sigma_constant: float,
            max_boxcar_width_in_sec: float, candidate_algorithm: int = 0, enable_msd_baseline_noise: bool = False,
            max_candidates: int | None = None, stream: int = 0) -> dict:
        """Candidates of one plane as numpy arrays: dm (trial index), ts
        (sample), snr, bw (boxcar width in samples of the range).
        max_candidates sizes the host lists (default: half the plane, at most
        2^24); a batch that would fill them is dropped, as in the reference."""
        import numpy as np
        ptr = d_plane if isinstance(d_plane, int) else d_plane.data_ptr()
        cap = (int(max_candidates) if max_candidates is not None
               else max(1, min(int(ndms) * int(nt) // 2, 1 << 24)))
        dm = np.zeros(cap, np.uint32)
        ts = np.zeros(cap, np.uint32)
        snr = np.zeros(cap, np.float32)
        bw = np.zeros(cap, np.uint32)
        n = ctypes.c_size_t()
        rc = lib().aa_b200_spd_run(self.m_obj, ctypes.c_void_p(ptr), int(ndms), int(nt), float(tsamp), int(inBin),
                                   float(sigma_cutoff), float(sigma_constant), float(max_boxcar_width_in_sec),
                                   int(candidate_algorithm), int(bool(enable_msd_baseline_noise)),
                                   ctypes.c_void_p(stream), cap, dm.ctypes.data, ts.ctypes.data, snr.ctypes.data,
                                   bw.ctypes.data, ctypes.byref(n))
        if rc:
            raise RuntimeError(self.last_error())
        k = n.value
        return {"dm": dm[:k].copy(), "ts": ts[:k].copy(), "snr": snr[:k].copy(), "bw": bw[:k].copy()}

    def profile(self) -> dict:
        """The plan and the interpolated (mean, deviation) per width of the last run."""
        import numpy as np
        cap = 1024
        msd = np.zeros(2 * cap, np.float32)
        widths = np.zeros(cap, np.int32)
        nw, mwp, mit, drop = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        lib().aa_b200_spd_profile(self.m_obj, msd.ctypes.data, cap, widths.ctypes.data, ctypes.byref(nw),
                                  ctypes.byref(mwp), ctypes.byref(mit), ctypes.byref(drop))
        k = nw.value
        return {"widths": widths[:k].copy(), "msd": msd[:2 * k].copy(), "max_width_performed": mwp.value,
                "max_iteration": mit.value, "dropped_batches": drop.value}

    def time_kernels(self, on: bool = True):
        lib().aa_b200_spd_time_kernels(self.m_obj, int(on))

    def msd_profile(self, d_plane, ndms: int, nt: int, widths, high_memory: bool = False,
                    sigma_constant: float = 3.0, outlier_rejection: bool = False, stream: int = 0):
        """(mean, deviation) per width of the MSD plane profile, float32 [2*len(widths)]."""
        w = np.ascontiguousarray(widths, np.int32)
        out = np.zeros(2 * w.size, np.float32)
        ptr = d_plane if isinstance(d_plane, int) else d_plane.data_ptr()
        if lib().aa_b200_spd_msd_profile(self.m_obj, ctypes.c_void_p(ptr), int(ndms), int(nt),
                                         w.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), w.size, int(high_memory),
                                         float(sigma_constant), int(outlier_rejection), out.ctypes.data,
                                         ctypes.c_void_p(stream)):
            raise RuntimeError(self.last_error())
        return out

    def family_times(self) -> dict:
        """Device ms and launches per launch family of the last run (time_kernels on)."""
        out = {}
        for k, name in enumerate(("msd", "decimation", "snr_first", "snr_later", "candidates")):
            ms, n = ctypes.c_double(), ctypes.c_longlong()
            lib().aa_b200_spd_family_time(self.m_obj, k, ctypes.byref(ms), ctypes.byref(n))
            out[name] = (ms.value, n.value)
        return out

    def planes(self):
        """(snr, taps) of the last batch of the last run (keep_planes on)."""
        import numpy as np
        n = lib().aa_b200_spd_planes(self.m_obj, None, None, 0)
        snr = np.zeros(n, np.float32)
        taps = np.zeros(n, np.uint16)
        lib().aa_b200_spd_planes(self.m_obj, snr.ctypes.data, taps.ctypes.data, n)
        return snr, taps

    def delete(self):
        if getattr(self, "m_obj", None):
            lib().aa_b200_spd_destroy(self.m_obj)
            self.m_obj = None

    def __del__(self):
        try:
            self.delete()
        except Exception:
            pass


def spd_plan(nt: int, tsamp: float, inBin: int, max_boxcar_width_in_sec: float) -> dict:
    """The boxcar plan of the single-pulse detection (host only)."""
    w = np.zeros(1024, np.int32)
    pl = np.zeros(10 * 64, np.int32)
    nw, mwp, mit, npl = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    if lib().aa_b200_spd_plan(int(nt), float(tsamp), int(inBin), float(max_boxcar_width_in_sec), w.ctypes.data,
                              1024, ctypes.byref(nw), ctypes.byref(mwp), ctypes.byref(mit), pl.ctypes.data, 64,
                              ctypes.byref(npl)):
        raise ValueError(lib().aa_b200_spd_last_error(None).decode())
    return {"widths": w[:nw.value].tolist(), "max_width_performed": mwp.value, "max_iteration": mit.value,
            "plan": pl[:10 * npl.value].reshape(-1, 10).tolist()}


def spd_kernel_launches() -> int:
    return lib().aa_b200_spd_kernel_launches()


def tuned_ranges(clear: bool = False) -> int:
    """Autotuner choices kept in this process (one per distinct range shape;
    a later pipeline of the same shape reuses them); clear drops them first."""
    return int(lib().aa_b200_tuned_ranges(1 if clear else 0))


def tuned_ranges_used() -> int:
    """Ranges set up from a kept autotuner choice in this process (not timed)."""
    return int(lib().aa_b200_tuned_ranges_used())


def save_tuned_ranges(path: str) -> int:
    """Write the kept autotuner choices to a text file; returns the entries."""
    n = lib().aa_b200_tuned_ranges_save(os.fsencode(path))
    if n < 0:
        raise OSError(lib().aa_b200_tuned_ranges_last_error().decode())
    return int(n)


def load_tuned_ranges(path: str) -> int:
    """Add the choices of a file written by save_tuned_ranges; returns the
    entries read."""
    n = lib().aa_b200_tuned_ranges_load(os.fsencode(path))
    if n < 0:
        raise OSError(lib().aa_b200_tuned_ranges_last_error().decode())
    return int(n)


def write_candidates(directory: str, candidate_algorithm: int, tstart: float, dm_low: float, dm_high: float,
                     dm_step: float, tsamp: float, inBin: int, cands: dict) -> None:
    """The reference's candidate file (peak_analysed-/analysed-t_..-dm_..-...dat)."""
    import numpy as np
    dm = np.ascontiguousarray(cands["dm"], np.uint32)
    ts = np.ascontiguousarray(cands["ts"], np.uint32)
    snr = np.ascontiguousarray(cands["snr"], np.float32)
    bw = np.ascontiguousarray(cands["bw"], np.uint32)
    if lib().aa_b200_spd_write_candidates(directory.encode() if directory else None, int(candidate_algorithm),
                                          float(tstart), float(dm_low), float(dm_high), float(dm_step),
                                          float(tsamp), int(inBin), dm.ctypes.data, ts.ctypes.data,
                                          snr.ctypes.data, bw.ctypes.data, dm.size):
        raise RuntimeError(lib().aa_b200_spd_last_error(None).decode())
