"""B200-native Lenia field update -- Python binding of the C ABI.

This package is a drop-in for the Lenia module step of LifeSimSuite
(daitomanabe/life-simulation, ``Modules/FieldModules/Lenia.{h,cpp}`` behind
``LifeCore/Sim/SimulationModule.h``). The compute path is the CUDA library
``liblenia_b200.so`` built from ``csrc/`` for sm_100a; this module only binds
its ``extern "C"`` entry points (``include/lenia_b200.h``) with ctypes and
mirrors the reference module's lifecycle::

    m = LeniaModule(params, scene_w, scene_h)   # configure + setup
    m.reset(seed)                               # reset
    m.encode(frame_index, substeps)             # updateCPU + encode
    a = m.field()                               # outputField (download)

There is no CPU fallback: importing the binding raises if the library is
missing, and every call raises ``LeniaError`` on a failed status.
"""
from __future__ import annotations

import ctypes
import json
import os
from typing import Optional, Sequence

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "liblenia_b200.so")

LENIA_OK = 0
LENIA_WARN_FALLBACK = 1
CONV_DIRECT, CONV_FFT, CONV_DIRECT_MULTI = 0, 1, 2
CORE_GAUSS_SHELL, CORE_EXP = 0, 1
FFT_FP32, FFT_BF16X3, FFT_FP16X3 = 0, 1, 2
ROWS_PIPELINED = 0x100  # rows-per-CTA flag of the software-pipelined row pass
COLS_HALF_THREADS = 0x40  # columns-per-CTA flag: half the threads, two last-pass items each
INIT_NOISE, INIT_STAMP = 0, 1


class LeniaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"lenia status {status}: {message}")
        self.status = status


class KernelDef(ctypes.Structure):
    """lenia_kernel_def (one entry of the scene "kernels" array)."""
    _fields_ = [("radius_scale", ctypes.c_float), ("mu", ctypes.c_float),
                ("sigma", ctypes.c_float), ("weight", ctypes.c_float),
                ("num_betas", ctypes.c_uint32), ("betas", ctypes.c_float * 8)]


class Config(ctypes.Structure):
    """lenia_config (the scene "params" block, parsed)."""
    _fields_ = [("sim_width", ctypes.c_uint32), ("sim_height", ctypes.c_uint32),
                ("conv_mode", ctypes.c_uint32), ("fft_any_size", ctypes.c_uint32),
                ("has_radius", ctypes.c_uint32), ("radius", ctypes.c_uint32),
                ("num_kernels", ctypes.c_uint32), ("kernels", KernelDef * 4),
                ("kernel_core", ctypes.c_uint32), ("kernel_shell_mu", ctypes.c_float),
                ("kernel_shell_sigma", ctypes.c_float), ("init_coverage", ctypes.c_float),
                ("init_scale", ctypes.c_float), ("init_mode", ctypes.c_uint32),
                ("organism_cells", ctypes.POINTER(ctypes.c_float)),
                ("org_width", ctypes.c_uint32), ("org_height", ctypes.c_uint32),
                ("org_R", ctypes.c_float), ("org_T", ctypes.c_float),
                ("org_mu", ctypes.c_float), ("org_sigma", ctypes.c_float),
                ("stamp_count", ctypes.c_uint32), ("stamp_rotate", ctypes.c_uint32),
                ("use_organism_params", ctypes.c_uint32), ("fft_precision", ctypes.c_uint32)]


class FrameParams(ctypes.Structure):
    """lenia_frame_params (the per-frame param() values)."""
    _fields_ = [("dt", ctypes.c_float), ("growth_mu", ctypes.c_float),
                ("growth_sigma", ctypes.c_float), ("noise_amount", ctypes.c_float),
                ("mu_jitter", ctypes.c_float), ("inject_amount", ctypes.c_float),
                ("inject_count", ctypes.c_uint32), ("growth_mode", ctypes.c_uint32),
                ("frame_index", ctypes.c_uint32), ("audio_frame", ctypes.c_uint32)]


class Info(ctypes.Structure):
    _fields_ = [("sim_width", ctypes.c_uint32), ("sim_height", ctypes.c_uint32),
                ("conv_mode", ctypes.c_uint32), ("radius", ctypes.c_uint32),
                ("num_kernels", ctypes.c_uint32), ("use_stamp_init", ctypes.c_uint32),
                ("device_bytes", ctypes.c_uint64), ("fft_radix_row", ctypes.c_uint32 * 8),
                ("fft_radix_col", ctypes.c_uint32 * 8), ("fft_precision", ctypes.c_uint32),
                ("direct_tma", ctypes.c_uint32), ("direct_split", ctypes.c_uint32),
                ("direct_outputs_per_thread", ctypes.c_uint32), ("direct_taps", ctypes.c_uint32),
                ("direct_rows_per_thread", ctypes.c_uint32), ("tc_engine", ctypes.c_uint32)]


# Every symbol include/lenia_b200.h declares (checked by the CPU tests).
EXPORTS = (
    "lenia_config_defaults", "lenia_create", "lenia_create_json", "lenia_inspect_json",
    "lenia_destroy",
    "lenia_reset", "lenia_set_param", "lenia_set_override", "lenia_clear_override",
    "lenia_resolve_frame_params", "lenia_encode", "lenia_step", "lenia_sync",
    "lenia_field_size", "lenia_upload", "lenia_download", "lenia_upload_device",
    "lenia_download_device", "lenia_field_device_ptr", "lenia_get_info",
    "lenia_get_stream", "lenia_profile", "lenia_profile_read", "lenia_get_tuning", "lenia_set_tuning",
    "lenia_last_message", "lenia_status_string",
    "lenia_fft_step_noalloc", "lenia_noalloc_last_message", "lenia_fp32_peak",
    "lenia_batch_create", "lenia_batch_destroy", "lenia_batch_upload", "lenia_batch_download",
    "lenia_batch_step", "lenia_batch_stats", "lenia_batch_world_path", "lenia_batch_sync",
    "lenia_batch_last_message",
    "lenia_adjoint_create", "lenia_adjoint_destroy", "lenia_adjoint_set_params",
    "lenia_adjoint_forward", "lenia_adjoint_backward", "lenia_adjoint_stats",
    "lenia_adjoint_last_message",
    "lenia_bus_create", "lenia_bus_destroy", "lenia_bus_load_scene", "lenia_bus_add_mapping",
    "lenia_bus_set_base", "lenia_bus_set_override", "lenia_bus_clear_override", "lenia_bus_set_feature",
    "lenia_bus_set_section", "lenia_bus_clear_features", "lenia_bus_update", "lenia_bus_value",
    "lenia_bus_last_message", "lenia_create_scene_module", "lenia_attach_bus",
    "lenia_get_colormap", "lenia_set_colormap", "lenia_colormap_from_json", "lenia_render_rgba16f",
    "lenia_step_render",
    "lenia_batch_init_noise", "lenia_batch_activity", "lenia_batch_launch_form", "lenia_batch_set_launch_form",
    "lenia_npy_write_f32", "lenia_npy_read_f32", "lenia_save_state", "lenia_load_state",
)


class ColorMap(ctypes.Structure):
    """lenia_colormap (the module's cosine palette)."""
    _fields_ = [("a", ctypes.c_float * 3), ("b", ctypes.c_float * 3), ("c", ctypes.c_float * 3),
                ("d", ctypes.c_float * 3), ("input_scale", ctypes.c_float), ("input_bias", ctypes.c_float),
                ("exposure", ctypes.c_float), ("channel", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        return {"a": list(self.a), "b": list(self.b), "c": list(self.c), "d": list(self.d),
                "inputScale": self.input_scale, "inputBias": self.input_bias, "exposure": self.exposure,
                "channel": self.channel}

MAP_ADD, MAP_SET, MAP_MUL = 0, 1, 2


class Mapping(ctypes.Structure):
    """lenia_mapping (one audio/music/automation mapping)."""
    _fields_ = [("source", ctypes.c_char_p), ("target", ctypes.c_char_p), ("in_min", ctypes.c_float),
                ("in_max", ctypes.c_float), ("scale", ctypes.c_float), ("offset", ctypes.c_float),
                ("smoothing", ctypes.c_float), ("mode", ctypes.c_uint32)]


class SceneInfo(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint32), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("num_modules", ctypes.c_uint32), ("num_mappings", ctypes.c_uint32)]

ADJOINT_PARAMS_PER_KERNEL = 11
ADJOINT_NUM_PARAMS = 45


class AdjointConfig(ctypes.Structure):
    """lenia_adjoint_config (a batch of worlds for gradient computation)."""
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("batch", ctypes.c_uint32),
                ("radius", ctypes.c_uint32), ("kernel_core", ctypes.c_uint32), ("shell_sigma", ctypes.c_float),
                ("growth_mode", ctypes.c_uint32), ("dt", ctypes.c_float), ("num_kernels", ctypes.c_uint32),
                ("kernels", KernelDef * 4), ("steps", ctypes.c_uint32), ("checkpoint_every", ctypes.c_uint32)]

BATCH_AUTO, BATCH_DIRECT, BATCH_FFT = 0, 1, 2
BATCH_FORM_PER_SIZE, BATCH_FORM_PERSISTENT = 0, 1


class World(ctypes.Structure):
    """lenia_world: one world of a batch (single-ring Lenia)."""
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("radius", ctypes.c_uint32),
                ("mu", ctypes.c_float), ("sigma", ctypes.c_float), ("dt", ctypes.c_float),
                ("growth_mode", ctypes.c_uint32), ("kernel_core", ctypes.c_uint32),
                ("shell_mu", ctypes.c_float), ("shell_sigma", ctypes.c_float), ("seed", ctypes.c_uint32)]

PHASES = ("init", "direct", "row_fft", "column", "row_growth", "colormap")


class ProfileData(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_uint64), ("count", ctypes.c_uint32 * 8),
                ("ms", ctypes.c_double * 8)]

_LIB = None


def load_library(path: str = LIB_PATH):
    """Loads liblenia_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m life_simulation_b200.build`")
    L = ctypes.CDLL(path)
    P, u32, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int
    pp = ctypes.POINTER(ctypes.c_void_p)
    L.lenia_config_defaults.argtypes = [ctypes.POINTER(Config)]
    L.lenia_config_defaults.restype = None
    L.lenia_create.argtypes = [ctypes.POINTER(Config), u32, u32, pp]
    L.lenia_create_json.argtypes = [ctypes.c_char_p, u32, u32, ctypes.c_char_p, pp]
    L.lenia_inspect_json.argtypes = [ctypes.c_char_p, u32, u32, ctypes.c_char_p, ctypes.POINTER(Info)]
    L.lenia_destroy.argtypes = [P]
    L.lenia_reset.argtypes = [P, u32]
    L.lenia_set_param.argtypes = [P, ctypes.c_char_p, ctypes.c_float]
    L.lenia_set_override.argtypes = [P, ctypes.c_char_p, ctypes.c_float]
    L.lenia_clear_override.argtypes = [P, ctypes.c_char_p]
    L.lenia_resolve_frame_params.argtypes = [P, u32, u32, ctypes.POINTER(FrameParams)]
    L.lenia_encode.argtypes = [P, u32, u32, u32, P]
    L.lenia_step.argtypes = [P, ctypes.POINTER(FrameParams), u32, P]
    L.lenia_sync.argtypes = [P]
    L.lenia_field_size.argtypes = [P, ctypes.POINTER(u32), ctypes.POINTER(u32)]
    L.lenia_upload.argtypes = [P, P, ctypes.c_size_t]
    L.lenia_download.argtypes = [P, P, ctypes.c_size_t]
    L.lenia_upload_device.argtypes = [P, P, ctypes.c_size_t, P]
    L.lenia_download_device.argtypes = [P, P, ctypes.c_size_t, P]
    L.lenia_field_device_ptr.argtypes = [P, pp]
    L.lenia_get_info.argtypes = [P, ctypes.POINTER(Info)]
    L.lenia_get_stream.argtypes = [P, pp]
    L.lenia_profile.argtypes = [P, i32]
    L.lenia_profile_read.argtypes = [P, ctypes.POINTER(ProfileData)]
    L.lenia_get_tuning.argtypes = [P, ctypes.POINTER(i32), ctypes.POINTER(i32)]
    L.lenia_set_tuning.argtypes = [P, i32, i32]
    L.lenia_last_message.argtypes = [P]
    L.lenia_last_message.restype = ctypes.c_char_p
    L.lenia_status_string.argtypes = [i32]
    L.lenia_status_string.restype = ctypes.c_char_p
    L.lenia_fft_step_noalloc.argtypes = [P, P, u32, u32, ctypes.POINTER(Config),
                                         ctypes.POINTER(FrameParams), u32, P]
    L.lenia_noalloc_last_message.argtypes = []
    L.lenia_noalloc_last_message.restype = ctypes.c_char_p
    L.lenia_fp32_peak.argtypes = [i32, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), P]
    L.lenia_batch_create.argtypes = [ctypes.POINTER(World), u32, u32, pp]
    L.lenia_batch_destroy.argtypes = [P]
    L.lenia_batch_upload.argtypes = [P, u32, P]
    L.lenia_batch_download.argtypes = [P, u32, P]
    L.lenia_batch_step.argtypes = [P, u32, P]
    L.lenia_batch_stats.argtypes = [P, P, P]
    L.lenia_batch_world_path.argtypes = [P, u32, ctypes.POINTER(u32)]
    L.lenia_batch_sync.argtypes = [P]
    L.lenia_batch_last_message.argtypes = [P]
    L.lenia_batch_last_message.restype = ctypes.c_char_p
    L.lenia_adjoint_create.argtypes = [ctypes.POINTER(AdjointConfig), pp]
    L.lenia_adjoint_destroy.argtypes = [P]
    L.lenia_adjoint_set_params.argtypes = [P, ctypes.POINTER(KernelDef), u32, ctypes.c_float]
    L.lenia_adjoint_forward.argtypes = [P, P, P, P]
    L.lenia_adjoint_backward.argtypes = [P, P, P, P, P]
    L.lenia_adjoint_stats.argtypes = [P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    L.lenia_adjoint_last_message.argtypes = [P]
    L.lenia_adjoint_last_message.restype = ctypes.c_char_p
    L.lenia_bus_create.argtypes = [u32, pp]
    L.lenia_bus_destroy.argtypes = [P]
    L.lenia_bus_load_scene.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(SceneInfo)]
    L.lenia_bus_add_mapping.argtypes = [P, ctypes.POINTER(Mapping)]
    L.lenia_bus_set_base.argtypes = [P, ctypes.c_char_p, ctypes.c_float]
    L.lenia_bus_set_override.argtypes = [P, ctypes.c_char_p, ctypes.c_float]
    L.lenia_bus_clear_override.argtypes = [P, ctypes.c_char_p]
    L.lenia_bus_set_feature.argtypes = [P, ctypes.c_char_p, ctypes.c_float]
    L.lenia_bus_set_section.argtypes = [P, ctypes.c_char_p, ctypes.c_int32]
    L.lenia_bus_clear_features.argtypes = [P]
    L.lenia_bus_update.argtypes = [P, ctypes.c_float]
    L.lenia_bus_value.argtypes = [P, ctypes.c_char_p, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]
    L.lenia_bus_last_message.argtypes = [P]
    L.lenia_bus_last_message.restype = ctypes.c_char_p
    L.lenia_create_scene_module.argtypes = [ctypes.c_char_p, ctypes.c_char_p, P, ctypes.c_char_p, pp]
    L.lenia_attach_bus.argtypes = [P, P]
    L.lenia_get_colormap.argtypes = [P, ctypes.POINTER(ColorMap)]
    L.lenia_set_colormap.argtypes = [P, ctypes.POINTER(ColorMap)]
    L.lenia_colormap_from_json.argtypes = [ctypes.c_char_p, ctypes.POINTER(ColorMap)]
    L.lenia_render_rgba16f.argtypes = [P, P, u32, u32, P]
    L.lenia_step_render.argtypes = [P, ctypes.POINTER(FrameParams), u32, P, u32, u32, P]
    L.lenia_batch_init_noise.argtypes = [P, u32, u32, ctypes.c_float, ctypes.c_float]
    L.lenia_npy_write_f32.argtypes = [ctypes.c_char_p, P, ctypes.c_size_t, P, u32]
    L.lenia_npy_read_f32.argtypes = [ctypes.c_char_p, P, u32, P, ctypes.c_size_t]
    L.lenia_save_state.argtypes = [P, ctypes.c_char_p]
    L.lenia_load_state.argtypes = [P, ctypes.c_char_p]
    L.lenia_batch_activity.argtypes = [P, ctypes.POINTER(ColorMap), P, P]
    L.lenia_batch_launch_form.argtypes = [P, ctypes.POINTER(u32)]
    L.lenia_batch_set_launch_form.argtypes = [P, u32]
    for name in EXPORTS:
        getattr(L, name)  # raises AttributeError if the build lacks a symbol
    _LIB = L
    return L


def default_config() -> Config:
    c = Config()
    load_library().lenia_config_defaults(ctypes.byref(c))
    return c


def config_from_params(params: dict) -> Config:
    """A lenia_config from a scene ``params`` dict (organism given as cells)."""
    c = default_config()
    c.sim_width = int(params.get("simWidth", 0))
    c.sim_height = int(params.get("simHeight", 0))
    c.conv_mode = {"fft": CONV_FFT, "directMulti": CONV_DIRECT_MULTI}.get(params.get("convMode", "direct"), CONV_DIRECT)
    c.fft_any_size = int(bool(params.get("fftAnySize", False)))
    c.fft_precision = {"fp32": FFT_FP32, "bf16x3": FFT_BF16X3, "fp16x3": FFT_FP16X3}[params.get("fftPrecision", "fp32")]
    if "radius" in params:
        c.has_radius, c.radius = 1, int(params["radius"])
    ks = params.get("kernels") or []
    c.num_kernels = len(ks)
    for i, k in enumerate(ks[:4]):
        b = list(k.get("betas") or [1.0])
        c.kernels[i].radius_scale = k.get("radiusScale", 1.0)
        c.kernels[i].mu = k.get("mu", 0.15)
        c.kernels[i].sigma = k.get("sigma", 0.017)
        c.kernels[i].weight = k.get("weight", 1.0)
        c.kernels[i].num_betas = len(b)
        for j, v in enumerate(b[:8]):
            c.kernels[i].betas[j] = v
    c.kernel_core = CORE_EXP if params.get("kernelCore", "gaussShell") == "exp" else CORE_GAUSS_SHELL
    c.kernel_shell_mu = params.get("kernelShellMu", 0.5)
    c.kernel_shell_sigma = params.get("kernelShellSigma", 0.15)
    c.init_coverage = params.get("initCoverage", 0.4)
    c.init_scale = params.get("initScale", 24.0)
    c.init_mode = INIT_STAMP if params.get("initMode", "noise") == "stamp" else INIT_NOISE
    c.stamp_count = min(32, int(params.get("stampCount", 6)))
    c.stamp_rotate = int(bool(params.get("stampRotate", True)))
    c.use_organism_params = int(bool(params.get("useOrganismParams", True)))
    return c


class LeniaModule:
    """The reference LeniaModule's lifecycle over the CUDA library.

    ``params``: the module's scene ``params`` dict (or its JSON text), exactly
    as in the reference presets; ``scene_w``/``scene_h``: the scene size
    (``SimulationContext::width/height``). ``base_dir`` resolves a relative
    ``organism`` path. A setup fallback of the reference is not an error:
    ``self.warning`` holds its message.
    """

    def __init__(self, params, scene_w: int, scene_h: int, base_dir: Optional[str] = None):
        L = load_library()
        self._L = L
        self._h = ctypes.c_void_p()
        text = params if isinstance(params, str) else json.dumps(params)
        rc = L.lenia_create_json(text.encode(), scene_w, scene_h,
                                 base_dir.encode() if base_dir else None, ctypes.byref(self._h))
        if rc < 0:
            raise LeniaError(rc, L.lenia_last_message(None).decode(errors="replace"))
        self.warning = L.lenia_last_message(self._h).decode(errors="replace") if rc > 0 else ""
        w, h = ctypes.c_uint32(), ctypes.c_uint32()
        self._check(L.lenia_field_size(self._h, ctypes.byref(w), ctypes.byref(h)))
        self.width, self.height = w.value, h.value

    @classmethod
    def from_config(cls, cfg: Config, scene_w: int, scene_h: int) -> "LeniaModule":
        self = cls.__new__(cls)
        L = load_library()
        self._L = L
        self._h = ctypes.c_void_p()
        rc = L.lenia_create(ctypes.byref(cfg), scene_w, scene_h, ctypes.byref(self._h))
        if rc < 0:
            raise LeniaError(rc, L.lenia_last_message(None).decode(errors="replace"))
        self.warning = L.lenia_last_message(self._h).decode(errors="replace") if rc > 0 else ""
        w, h = ctypes.c_uint32(), ctypes.c_uint32()
        self._check(L.lenia_field_size(self._h, ctypes.byref(w), ctypes.byref(h)))
        self.width, self.height = w.value, h.value
        return self

    def _check(self, rc: int) -> int:
        if rc < 0:
            msg = self._L.lenia_last_message(self._h).decode(errors="replace")
            raise LeniaError(rc, msg or self._L.lenia_status_string(rc).decode())
        return rc

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._L.lenia_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self, seed: int) -> None:
        self._check(self._L.lenia_reset(self._h, seed & 0xFFFFFFFF))

    def set_param(self, key: str, value: float) -> None:
        self._check(self._L.lenia_set_param(self._h, key.encode(), value))

    def set_override(self, key: str, value: float) -> None:
        self._check(self._L.lenia_set_override(self._h, key.encode(), value))

    def clear_override(self, key: str) -> None:
        self._check(self._L.lenia_clear_override(self._h, key.encode()))

    def frame_params(self, frame_index: int = 0, audio_frame: Optional[int] = None) -> FrameParams:
        fp = FrameParams()
        af = frame_index if audio_frame is None else audio_frame
        self._check(self._L.lenia_resolve_frame_params(self._h, frame_index, af, ctypes.byref(fp)))
        return fp

    def encode(self, frame_index: int, substeps: int = 1, audio_frame: Optional[int] = None,
               stream: Optional[int] = None) -> None:
        af = frame_index if audio_frame is None else audio_frame
        self._check(self._L.lenia_encode(self._h, frame_index, substeps, af,
                                         ctypes.c_void_p(stream) if stream else None))

    def step(self, fp: FrameParams, substeps: int = 1, stream: Optional[int] = None) -> None:
        self._check(self._L.lenia_step(self._h, ctypes.byref(fp), substeps,
                                       ctypes.c_void_p(stream) if stream else None))

    def sync(self) -> None:
        self._check(self._L.lenia_sync(self._h))

    def field(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        self._check(self._L.lenia_download(self._h, out.ctypes.data_as(ctypes.c_void_p), out.size))
        return out

    def download_into(self, out: np.ndarray) -> np.ndarray:
        """Downloads the field into a caller buffer (e.g. pinned memory)."""
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.size != self.width * self.height:
            raise ValueError("out must be a contiguous float32 array of the field's size")
        self._check(self._L.lenia_download(self._h, out.ctypes.data_as(ctypes.c_void_p), out.size))
        return out

    def upload(self, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, np.float32)
        if a.size != self.width * self.height:
            raise ValueError("field size mismatch")
        self._check(self._L.lenia_upload(self._h, a.ctypes.data_as(ctypes.c_void_p), a.size))

    def upload_device(self, ptr: int, stream: Optional[int] = None) -> None:
        self._check(self._L.lenia_upload_device(self._h, ctypes.c_void_p(ptr), self.width * self.height,
                                                ctypes.c_void_p(stream) if stream else None))

    def download_device(self, ptr: int, stream: Optional[int] = None) -> None:
        self._check(self._L.lenia_download_device(self._h, ctypes.c_void_p(ptr), self.width * self.height,
                                                  ctypes.c_void_p(stream) if stream else None))

    def colormap(self) -> ColorMap:
        cm = ColorMap()
        self._check(self._L.lenia_get_colormap(self._h, ctypes.byref(cm)))
        return cm

    def set_colormap(self, cm: ColorMap) -> None:
        self._check(self._L.lenia_set_colormap(self._h, ctypes.byref(cm)))

    def render_device(self, ptr: int, width: int, height: int, stream: Optional[int] = None) -> None:
        """Colour layer (RGBA16F, 8 bytes per pixel) into a device buffer."""
        self._check(self._L.lenia_render_rgba16f(self._h, ctypes.c_void_p(ptr), width, height,
                                                 ctypes.c_void_p(stream) if stream else None))

    def step_render(self, fp: "FrameParams", substeps: int, ptr: int, width: int, height: int,
                    stream: Optional[int] = None) -> None:
        """step() then the colour layer of the new field into a device
        buffer; at the sim size on the spectral path the last substep writes
        it directly (no separate colour pass). Same texels as render_device."""
        self._check(self._L.lenia_step_render(self._h, ctypes.byref(fp), substeps, ctypes.c_void_p(ptr), width,
                                              height, ctypes.c_void_p(stream) if stream else None))

    def save_state(self, path: str) -> None:
        """The field as a (height, width) float32 .npy file."""
        self._check(self._L.lenia_save_state(self._h, os.fsencode(path)))

    def load_state(self, path: str) -> None:
        """Replace the field from a (height, width) float32 .npy file."""
        self._check(self._L.lenia_load_state(self._h, os.fsencode(path)))

    def attach_bus(self, bus) -> None:
        """Read per-frame parameters from a shared ParamBus (None: own bus)."""
        self._check(self._L.lenia_attach_bus(self._h, bus._h if bus else None))
        self._bus = bus

    def field_device_ptr(self) -> int:
        p = ctypes.c_void_p()
        self._check(self._L.lenia_field_device_ptr(self._h, ctypes.byref(p)))
        return int(p.value or 0)

    def stream(self) -> int:
        """Handle of the context's own CUDA stream."""
        p = ctypes.c_void_p()
        self._check(self._L.lenia_get_stream(self._h, ctypes.byref(p)))
        return int(p.value or 0)

    def profile(self, enable: bool = True) -> None:
        """Starts (or stops) per-launch CUDA-event timing; resets counters."""
        self._check(self._L.lenia_profile(self._h, int(enable)))

    def profile_read(self) -> dict:
        """Device ms and launches per phase since the last read."""
        d = ProfileData()
        self._check(self._L.lenia_profile_read(self._h, ctypes.byref(d)))
        out = {"launches": int(d.launches)}
        for i, name in enumerate(PHASES):
            out[name] = {"count": int(d.count[i]), "ms": float(d.ms[i])}
        return out

    def tuning(self) -> tuple:
        """(columns per CTA, rows per CTA) of the spectral passes as tuned
        at setup (rows may carry ROWS_PIPELINED); (0, 0) without them."""
        c, r = ctypes.c_int32(), ctypes.c_int32()
        self._check(self._L.lenia_get_tuning(self._h, ctypes.byref(c), ctypes.byref(r)))
        return c.value, r.value

    def set_tuning(self, cols_per_cta: int, rows_per_cta: int) -> None:
        """Replaces the tuned launch shapes until the next setup."""
        self._check(self._L.lenia_set_tuning(self._h, int(cols_per_cta), int(rows_per_cta)))

    def info(self) -> dict:
        i = Info()
        self._check(self._L.lenia_get_info(self._h, ctypes.byref(i)))
        return {"sim_width": i.sim_width, "sim_height": i.sim_height, "conv_mode": i.conv_mode,
                "radius": i.radius, "num_kernels": i.num_kernels, "use_stamp_init": i.use_stamp_init,
                "device_bytes": i.device_bytes,
                "fft_radix_row": [r for r in i.fft_radix_row if r],
                "fft_radix_col": [r for r in i.fft_radix_col if r], "fft_precision": i.fft_precision,
                "direct_tma": bool(i.direct_tma), "direct_split": i.direct_split,
                "direct_outputs_per_thread": i.direct_outputs_per_thread, "direct_taps": i.direct_taps,
                "direct_rows_per_thread": i.direct_rows_per_thread, "tc_engine": i.tc_engine}


def inspect(params, scene_w: int, scene_h: int, base_dir: Optional[str] = None) -> dict:
    """What setup would resolve for these params, without a device
    (``lenia_inspect_json``): sizes, the path after the reference's
    fallbacks, radius, kernel count, FFT plans, and ``warning``."""
    L = load_library()
    text = params if isinstance(params, str) else json.dumps(params)
    i = Info()
    rc = L.lenia_inspect_json(text.encode(), scene_w, scene_h,
                              base_dir.encode() if base_dir else None, ctypes.byref(i))
    msg = L.lenia_last_message(None).decode(errors="replace")
    if rc < 0:
        raise LeniaError(rc, msg)
    return {"sim_width": i.sim_width, "sim_height": i.sim_height, "conv_mode": i.conv_mode,
            "radius": i.radius, "num_kernels": i.num_kernels, "use_stamp_init": i.use_stamp_init,
            "fft_radix_row": [r for r in i.fft_radix_row if r],
            "fft_radix_col": [r for r in i.fft_radix_col if r],
            "status": rc, "warning": msg if rc > 0 else ""}


def fp32_peak(reps: int = 5, stream: Optional[int] = None) -> dict:
    """Measured FP32 FMA peak of the current device in TFLOP/s: scalar FFMA
    and packed FFMA2 (lenia_fp32_peak)."""
    L = load_library()
    a, b = ctypes.c_double(), ctypes.c_double()
    rc = L.lenia_fp32_peak(reps, ctypes.byref(a), ctypes.byref(b), ctypes.c_void_p(stream) if stream else None)
    if rc != 0:
        raise LeniaError(rc, "lenia_fp32_peak failed")
    return {"ffma_tflops": a.value, "ffma2_tflops": b.value}


def make_frame_params(dt=0.1, growth_mu=0.15, growth_sigma=0.017, noise_amount=0.0, mu_jitter=0.0,
                      inject_amount=0.0, inject_count=3, growth_mode=1, frame_index=0,
                      audio_frame=None) -> FrameParams:
    fp = FrameParams()
    fp.dt, fp.growth_mu, fp.growth_sigma = dt, growth_mu, growth_sigma
    fp.noise_amount, fp.mu_jitter, fp.inject_amount = noise_amount, mu_jitter, inject_amount
    fp.inject_count, fp.growth_mode = inject_count, growth_mode
    fp.frame_index = frame_index
    fp.audio_frame = frame_index if audio_frame is None else audio_frame
    return fp


def make_world(width, height, radius, mu, sigma, dt, growth_mode=0, kernel_core=CORE_GAUSS_SHELL,
               shell_mu=0.5, shell_sigma=0.15, seed=0) -> World:
    w = World()
    w.width, w.height, w.radius = width, height, radius
    w.mu, w.sigma, w.dt, w.growth_mode, w.kernel_core = mu, sigma, dt, growth_mode, kernel_core
    w.shell_mu, w.shell_sigma, w.seed = shell_mu, shell_sigma, seed
    return w


class LeniaBatch:
    """Many independent worlds stepped together (lenia_batch_*)."""

    def __init__(self, worlds, policy: int = BATCH_AUTO):
        L = load_library()
        self._L = L
        self.worlds = list(worlds)
        arr = (World * len(self.worlds))(*self.worlds)
        self._h = ctypes.c_void_p()
        rc = L.lenia_batch_create(arr, len(self.worlds), policy, ctypes.byref(self._h))
        if rc < 0:
            raise LeniaError(rc, "batch creation failed")

    def _check(self, rc: int) -> int:
        if rc < 0:
            raise LeniaError(rc, self._L.lenia_batch_last_message(self._h).decode(errors="replace"))
        return rc

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._L.lenia_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, i: int, a: np.ndarray) -> None:
        w = self.worlds[i]
        a = np.ascontiguousarray(a, np.float32)
        if a.size != w.width * w.height:
            raise ValueError("field size mismatch")
        self._check(self._L.lenia_batch_upload(self._h, i, a.ctypes.data_as(ctypes.c_void_p)))

    def field(self, i: int) -> np.ndarray:
        w = self.worlds[i]
        out = np.empty((w.height, w.width), np.float32)
        self._check(self._L.lenia_batch_download(self._h, i, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def step(self, steps: int = 1, stream: Optional[int] = None) -> None:
        self._check(self._L.lenia_batch_step(self._h, steps, ctypes.c_void_p(stream) if stream else None))

    def sync(self) -> None:
        self._check(self._L.lenia_batch_sync(self._h))

    def stats(self):
        n = len(self.worlds)
        mean = np.empty(n, np.float64)
        var = np.empty(n, np.float64)
        self._check(self._L.lenia_batch_stats(self._h, mean.ctypes.data_as(ctypes.c_void_p),
                                              var.ctypes.data_as(ctypes.c_void_p)))
        return mean, var

    def init_noise(self, i: int, seed: int, coverage: float = 0.4, scale: float = 24.0) -> None:
        """The reference module's noise init of world i (reset seed `seed`)."""
        self._check(self._L.lenia_batch_init_noise(self._h, i, seed, coverage, scale))

    def activity(self, cm: "ColorMap"):
        """Per-world mean and standard deviation of the colour layer's luma."""
        n = len(self.worlds)
        mean = np.empty(n, np.float64)
        std = np.empty(n, np.float64)
        self._check(self._L.lenia_batch_activity(self._h, ctypes.byref(cm), mean.ctypes.data_as(ctypes.c_void_p),
                                                 std.ctypes.data_as(ctypes.c_void_p)))
        return mean, std

    def path(self, i: int) -> int:
        p = ctypes.c_uint32()
        self._check(self._L.lenia_batch_world_path(self._h, i, ctypes.byref(p)))
        return p.value

    def launch_form(self) -> int:
        """BATCH_FORM_PERSISTENT (one launch per substep) or BATCH_FORM_PER_SIZE."""
        f = ctypes.c_uint32()
        self._check(self._L.lenia_batch_launch_form(self._h, ctypes.byref(f)))
        return f.value

    def set_launch_form(self, form: int) -> None:
        self._check(self._L.lenia_batch_set_launch_form(self._h, form))


def single_world_params(w: World, conv: str) -> dict:
    """Scene params of a single-world context equivalent to batch world `w`."""
    core = "exp" if w.kernel_core == CORE_EXP else "gaussShell"
    p = {"radius": int(w.radius), "dt": w.dt, "growthMu": w.mu, "growthSigma": w.sigma,
         "growthMode": int(w.growth_mode), "kernelCore": core, "kernelShellMu": w.shell_mu,
         "kernelShellSigma": w.shell_sigma, "noiseAmount": 0.0, "muJitter": 0.0, "injectAmount": 0.0}
    if conv == "fft":
        p.update(convMode="fft", fftAnySize=True,
                 kernels=[{"radiusScale": 1.0, "mu": w.mu, "sigma": w.sigma, "weight": 1.0, "betas": [1.0]}])
    return p


def kernel_defs(kernels) -> "ctypes.Array":
    """lenia_kernel_def[4] from dicts with mu, sigma, weight, betas and an
    optional radiusScale (the scene "kernels" entries)."""
    arr = (KernelDef * 4)()
    for i, k in enumerate(kernels):
        d = arr[i]
        d.radius_scale = float(k.get("radiusScale", 1.0))
        d.mu, d.sigma, d.weight = float(k["mu"]), float(k["sigma"]), float(k.get("weight", 1.0))
        betas = list(k.get("betas", [1.0]))
        d.num_betas = len(betas)
        for j, b in enumerate(betas):
            d.betas[j] = float(b)
    return arr


CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy


def _stream_arg(stream: Optional[int]):
    """None: the context's own stream (NULL); 0: the legacy default stream
    (torch's default stream reports handle 0); else the handle."""
    if stream is None:
        return None
    return ctypes.c_void_p(stream if stream else CUDA_STREAM_LEGACY)


class LeniaAdjoint:
    """Rollout and its gradient for a batch of worlds (lenia_adjoint_*).

    Device buffers are passed as integer device pointers (e.g. a torch
    tensor's data_ptr()): a0/a_final/g_final/g_initial hold batch x height x
    width float32 values; grad_params LENIA_ADJOINT_NUM_PARAMS float64.
    ``stream``: None queues on the context's own stream (ordered with
    nothing else: synchronise before touching the buffers); an int handle
    (0 = the legacy default stream, e.g. torch.cuda.current_stream()
    .cuda_stream) orders the work with that stream."""

    def __init__(self, width: int, height: int, batch: int, kernels, radius: int, steps: int,
                 checkpoint_every: Optional[int] = None, dt: float = 0.1, growth_mode: int = 0,
                 kernel_core: int = CORE_EXP, shell_sigma: float = 0.15):
        if checkpoint_every is None:
            checkpoint_every = min(8, steps)
        L = load_library()
        self._L = L
        c = AdjointConfig()
        c.width, c.height, c.batch, c.radius = width, height, batch, radius
        c.kernel_core, c.shell_sigma, c.growth_mode, c.dt = kernel_core, shell_sigma, growth_mode, dt
        c.num_kernels = len(kernels)
        c.kernels = kernel_defs(kernels)
        c.steps, c.checkpoint_every = steps, checkpoint_every
        self.config = c
        self.width, self.height, self.batch, self.steps = width, height, batch, steps
        self.num_kernels = len(kernels)
        self.num_betas = [len(k.get("betas", [1.0])) for k in kernels]
        self.radius_scales = [float(k.get("radiusScale", 1.0)) for k in kernels]
        self._h = ctypes.c_void_p()
        rc = L.lenia_adjoint_create(ctypes.byref(c), ctypes.byref(self._h))
        if rc < 0:
            raise LeniaError(rc, L.lenia_adjoint_last_message(None).decode(errors="replace"))
        self.forward_count = 0

    def _check(self, rc: int) -> int:
        if rc < 0:
            raise LeniaError(rc, self._L.lenia_adjoint_last_message(self._h).decode(errors="replace"))
        return rc

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._L.lenia_adjoint_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, kernels, dt: float) -> None:
        kd = kernel_defs([dict(k, radiusScale=s) for k, s in zip(kernels, self.radius_scales)])
        self._check(self._L.lenia_adjoint_set_params(self._h, kd, len(kernels), float(dt)))

    def forward(self, a0_ptr: int, out_ptr: int, stream: Optional[int] = None) -> None:
        self._check(self._L.lenia_adjoint_forward(self._h, ctypes.c_void_p(a0_ptr), ctypes.c_void_p(out_ptr),
                                                  _stream_arg(stream)))
        self.forward_count += 1

    def backward(self, g_final_ptr: int, g_initial_ptr: int, grad_params_ptr: Optional[int] = None,
                 stream: Optional[int] = None) -> None:
        self._check(self._L.lenia_adjoint_backward(
            self._h, ctypes.c_void_p(g_final_ptr), ctypes.c_void_p(g_initial_ptr),
            ctypes.c_void_p(grad_params_ptr) if grad_params_ptr else None, _stream_arg(stream)))

    def stats(self) -> dict:
        b = ctypes.c_uint64()
        n = ctypes.c_uint64()
        self._check(self._L.lenia_adjoint_stats(self._h, ctypes.byref(b), ctypes.byref(n)))
        return {"device_bytes": b.value, "launches": n.value}


def unpack_param_grads(g: Sequence[float], num_betas: Sequence[int]) -> dict:
    """The LENIA_ADJOINT_NUM_PARAMS gradient vector as per-kernel lists."""
    K = len(num_betas)
    per = ADJOINT_PARAMS_PER_KERNEL
    return {"mu": [g[k * per] for k in range(K)], "sigma": [g[k * per + 1] for k in range(K)],
            "weight": [g[k * per + 2] for k in range(K)],
            "betas": [[g[k * per + 3 + j] for j in range(num_betas[k])] for k in range(K)],
            "dt": g[ADJOINT_NUM_PARAMS - 1]}


class ParamBus:
    """The parameter bus (lenia_bus_*): bases, overrides, mappings from
    per-frame inputs and time sources, evaluated by update(dt). Host-only."""

    def __init__(self, seed: int = 0):
        L = load_library()
        self._L = L
        self._h = ctypes.c_void_p()
        rc = L.lenia_bus_create(seed, ctypes.byref(self._h))
        if rc < 0:
            raise LeniaError(rc, "bus creation failed")

    def _check(self, rc: int) -> int:
        if rc < 0:
            raise LeniaError(rc, self._L.lenia_bus_last_message(self._h).decode(errors="replace"))
        return rc

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._L.lenia_bus_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_scene(self, scene) -> dict:
        text = scene if isinstance(scene, str) else json.dumps(scene)
        info = SceneInfo()
        self._check(self._L.lenia_bus_load_scene(self._h, text.encode(), ctypes.byref(info)))
        return {"seed": info.seed, "width": info.width, "height": info.height,
                "num_modules": info.num_modules, "num_mappings": info.num_mappings}

    def add_mapping(self, source: str, target: str, in_min=0.0, in_max=0.0, scale=1.0, offset=0.0,
                    smoothing=0.0, mode: str = "add") -> None:
        m = Mapping(source.encode(), target.encode(), in_min, in_max, scale, offset, smoothing,
                    {"add": MAP_ADD, "set": MAP_SET, "mul": MAP_MUL, "multiply": MAP_MUL}.get(mode, MAP_ADD))
        self._check(self._L.lenia_bus_add_mapping(self._h, ctypes.byref(m)))

    def set_base(self, key: str, v: float) -> None:
        self._check(self._L.lenia_bus_set_base(self._h, key.encode(), v))

    def set_override(self, key: str, v: float) -> None:
        self._check(self._L.lenia_bus_set_override(self._h, key.encode(), v))

    def clear_override(self, key: str) -> None:
        self._check(self._L.lenia_bus_clear_override(self._h, key.encode()))

    def set_feature(self, name: str, v: float) -> None:
        self._check(self._L.lenia_bus_set_feature(self._h, name.encode(), v))

    def set_section(self, role: str, index: int) -> None:
        self._check(self._L.lenia_bus_set_section(self._h, role.encode(), index))

    def clear_features(self) -> None:
        self._check(self._L.lenia_bus_clear_features(self._h))

    def update(self, dt: float) -> None:
        self._check(self._L.lenia_bus_update(self._h, dt))

    def value(self, key: str, fallback: float = 0.0) -> float:
        out = ctypes.c_float()
        self._check(self._L.lenia_bus_value(self._h, key.encode(), fallback, ctypes.byref(out)))
        return out.value


def scene_module(scene, module_name: Optional[str] = None, bus: Optional[ParamBus] = None,
                 base_dir: Optional[str] = None) -> "LeniaModule":
    """The Lenia module of a scene document (lenia_create_scene_module)."""
    L = load_library()
    text = scene if isinstance(scene, str) else json.dumps(scene)
    m = LeniaModule.__new__(LeniaModule)
    m._L = L
    m._h = ctypes.c_void_p()
    rc = L.lenia_create_scene_module(text.encode(), module_name.encode() if module_name else None,
                                     bus._h if bus else None, base_dir.encode() if base_dir else None,
                                     ctypes.byref(m._h))
    if rc < 0:
        raise LeniaError(rc, L.lenia_last_message(None).decode(errors="replace"))
    m.warning = L.lenia_last_message(m._h).decode(errors="replace") if rc > 0 else ""
    m._bus = bus
    w, h = ctypes.c_uint32(), ctypes.c_uint32()
    m._check(L.lenia_field_size(m._h, ctypes.byref(w), ctypes.byref(h)))
    m.width, m.height = w.value, h.value
    return m


def colormap_from_params(params) -> ColorMap:
    """The palette a module's params give (no device)."""
    L = load_library()
    text = params if isinstance(params, str) else json.dumps(params)
    cm = ColorMap()
    rc = L.lenia_colormap_from_json(text.encode(), ctypes.byref(cm))
    if rc < 0:
        raise LeniaError(rc, L.lenia_last_message(None).decode(errors="replace"))
    return cm


def npy_write(path: str, a: np.ndarray) -> None:
    """A float32 array as a .npy v1.0 file (C order), by the library's writer."""
    L = load_library()
    a = np.ascontiguousarray(a, np.float32)
    shape = np.array(a.shape, np.uint32)
    rc = L.lenia_npy_write_f32(os.fsencode(path), a.ctypes.data_as(ctypes.c_void_p), a.size,
                               shape.ctypes.data_as(ctypes.c_void_p), a.ndim)
    if rc < 0:
        raise LeniaError(rc, L.lenia_last_message(None).decode(errors="replace"))


def npy_read(path: str, shape) -> np.ndarray:
    """A float32 .npy file that must have `shape`, by the library's reader."""
    L = load_library()
    shp = np.array(list(shape), np.uint32)
    out = np.empty(tuple(int(x) for x in shape), np.float32)
    rc = L.lenia_npy_read_f32(os.fsencode(path), shp.ctypes.data_as(ctypes.c_void_p), shp.size,
                              out.ctypes.data_as(ctypes.c_void_p), out.size)
    if rc < 0:
        raise LeniaError(rc, L.lenia_last_message(None).decode(errors="replace"))
    return out
