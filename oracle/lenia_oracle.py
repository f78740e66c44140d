"""CPU oracle for the Lenia field update -- TEST INFRASTRUCTURE ONLY.

This module is the oracle the CUDA path is compared against. Only tests/,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it; the product never does.

Three layers:

* ``lib()``: ctypes binding of ``oracle/_build/liblenia_oracle.so``, the C
  restatement of the reference's kernels (FP32 and FP64 builds of one source,
  ``oracle/lenia_oracle_body.h``).
* ``OracleLenia``: a restatement of the reference Lenia module's host logic
  (``Modules/FieldModules/Lenia.cpp``: setup 208-408, reset 448-451, encode
  455-644) over those kernels, in two precisions:
    - ``"ref32"`` reproduces the reference's FP32 arithmetic and pass order
      (direct sum order; radix-2 Stockham FFT with per-thread twiddles);
    - ``"f64"`` computes the same update in FP64 with exact circular
      convolution (numpy's float64 FFT of the kernel image), any field size.
* ``RefLenia``: ctypes binding of ``oracle/_ref/libleniaref.so``, the
  reference's own Metal kernels and ``Lenia.cpp`` compiled for the CPU (built
  only where the reference tree is present; used to pin the restatement).
"""
from __future__ import annotations

import ctypes
import json
import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liblenia_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libleniaref.so")

CORE_GAUSS_SHELL = 0
CORE_EXP = 1
LEN1_TAG = 0x4C454E31  # "LEN1", Lenia.cpp:449


class LoParams(ctypes.Structure):
    """LeniaParams, Shaders/Field/Lenia.metal:10-27."""

    _fields_ = [(n, ctypes.c_float) for n in (
        "dt", "growth_mu", "growth_sigma", "noise_amount", "mu_jitter",
        "init_coverage", "init_scale", "inject_amount")] + [
        (n, ctypes.c_uint32) for n in (
            "inject_count", "radius", "kernel_size", "seed", "width", "height",
            "frame_index", "growth_mode")]


class LoMultiParams(ctypes.Structure):
    """LeniaMultiParams, Shaders/Field/Lenia.metal:138-154."""

    _fields_ = [("dt", ctypes.c_float), ("k_mu", ctypes.c_float * 4),
                ("k_sigma", ctypes.c_float * 4), ("k_weight", ctypes.c_float * 4),
                ("num_kernels", ctypes.c_uint32), ("growth_mode", ctypes.c_uint32),
                ("noise_amount", ctypes.c_float), ("mu_jitter", ctypes.c_float),
                ("inject_amount", ctypes.c_float), ("inject_count", ctypes.c_uint32),
                ("radius", ctypes.c_uint32), ("seed", ctypes.c_uint32),
                ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("frame_index", ctypes.c_uint32)]


_LIB = None


def build_oracle() -> None:
    """Compiles the C restatement (gcc only)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    """The C restatement, built on first use."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = ctypes.CDLL(ORACLE_SO)
        P = ctypes.c_void_p
        u32, f32 = ctypes.c_uint32, ctypes.c_float
        L.lo_pcg_hash.restype = u32
        L.lo_pcg_hash.argtypes = [u32]
        L.lo_derive_seed.restype = u32
        L.lo_derive_seed.argtypes = [u32, u32]
        L.lo_rand01.restype = f32
        L.lo_rand01.argtypes = [u32, u32, u32, u32]
        L.lo_build_direct_lut.argtypes = [u32, f32, f32, ctypes.c_int, P]
        L.lo_build_ring_image.argtypes = [u32, u32, f32, f32, P, u32, ctypes.c_int, P]
        L.lo_init_noise.argtypes = [ctypes.POINTER(LoParams), P]
        L.lo_init_stamp.argtypes = [u32, u32, P, u32, u32, u32, u32, u32, P]
        L.lo_step_direct_f32.argtypes = [P, P, P, ctypes.POINTER(LoParams), u32]
        L.lo_step_direct_f64.argtypes = [P, P, P, ctypes.POINTER(LoParams), u32]
        L.lo_growth_multi_f32.argtypes = [P, P, P, ctypes.POINTER(LoMultiParams), u32]
        L.lo_growth_multi_f64.argtypes = [P, P, P, ctypes.POINTER(LoMultiParams), u32]
        L.lo_conv_direct_f64.argtypes = [P, P, u32, u32, P]
        L.lo_fft2d_ref_f32.argtypes = [P, P, u32, u32, ctypes.c_int]
        L.lo_step_fft_ref_f32.argtypes = [P, P, P, P, ctypes.POINTER(LoMultiParams), u32]
        _LIB = L
    return _LIB


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f32(x: float) -> float:
    return float(np.float32(x))


# ----------------------------------------------------------------- integer

def pcg_hash(v: int) -> int:
    """Shaders/Common/Random.metal:5-9."""
    return int(lib().lo_pcg_hash(v & 0xFFFFFFFF))


def derive_seed(seed: int, tag: int) -> int:
    """LifeCore/Math/Random.h:42-44."""
    return int(lib().lo_derive_seed(seed & 0xFFFFFFFF, tag & 0xFFFFFFFF))


def rand01(px: int, py: int, tag: int, seed: int) -> float:
    """Shaders/Common/Random.metal:16-19."""
    return float(lib().lo_rand01(px, py, tag, seed))


def pcg_hash_np(v: np.ndarray) -> np.ndarray:
    """Vectorised pcg_hash over uint32 arrays (same bit operations)."""
    v = v.astype(np.uint32)
    state = v * np.uint32(747796405) + np.uint32(2891336453)
    word = ((state >> ((state >> np.uint32(28)) + np.uint32(4))) ^ state) * np.uint32(277803737)
    return (word >> np.uint32(22)) ^ word


def rand01_np(px: np.ndarray, py: np.ndarray, tag: int, seed: int) -> np.ndarray:
    t = pcg_hash_np(np.array([(tag ^ seed) & 0xFFFFFFFF], np.uint32))[0]
    h = pcg_hash_np(px.astype(np.uint32) ^ pcg_hash_np(py.astype(np.uint32) ^ t))
    return (h >> np.uint32(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)


# ----------------------------------------------------- kernel construction

def direct_lut(radius: int, shell_mu: float = 0.5, shell_sigma: float = 0.15,
               core: int = CORE_GAUSS_SHELL) -> np.ndarray:
    """Lenia.cpp:410-446 (buildKernelTexture)."""
    size = 2 * radius + 1
    out = np.zeros((size, size), np.float32)
    lib().lo_build_direct_lut(radius, shell_mu, shell_sigma, core, _ptr(out))
    return out


def ring_image(w: int, h: int, radius_k: float, shell_sigma: float,
               betas: Sequence[float], core: int = CORE_GAUSS_SHELL) -> np.ndarray:
    """Lenia.cpp:95-125 (buildRingKernelImage), wrap-centred layout."""
    out = np.zeros((h, w), np.float32)
    b = np.ascontiguousarray(np.asarray(betas, np.float32))
    lib().lo_build_ring_image(w, h, radius_k, shell_sigma, _ptr(b), len(b), core, _ptr(out))
    return out


def fft2d_ref_f32(re: np.ndarray, im: np.ndarray, direction: int):
    """FFT.metal:65-121 driven as Lenia.cpp:57-85 (pow2 sizes only)."""
    re = np.ascontiguousarray(re, np.float32).copy()
    im = np.ascontiguousarray(im, np.float32).copy()
    h, w = re.shape
    lib().lo_fft2d_ref_f32(_ptr(re), _ptr(im), w, h, direction)
    return re, im


def conv_circular_f64(a: np.ndarray, kimg: np.ndarray) -> np.ndarray:
    """Exact (FP64) circular convolution of the field with a wrap-centred
    kernel image, pot[n] = sum_d K[d] A[n-d], via numpy's float64 FFT."""
    fa = np.fft.rfft2(np.asarray(a, np.float64))
    fk = np.fft.rfft2(np.asarray(kimg, np.float64))
    return np.fft.irfft2(fa * fk, s=a.shape)


def conv_direct_f64(a: np.ndarray, kimg: np.ndarray) -> np.ndarray:
    """Same convolution summed tap by tap in C (slow; small fields)."""
    a = np.ascontiguousarray(a, np.float64)
    k = np.ascontiguousarray(kimg, np.float32)
    h, w = a.shape
    out = np.zeros_like(a)
    lib().lo_conv_direct_f64(_ptr(a), _ptr(k), w, h, _ptr(out))
    return out


# -------------------------------------------------------------- module

@dataclass
class KernelDef:
    """Lenia.h:99-105 (one entry of the scene "kernels" array)."""
    radius_scale: float = 1.0
    mu: float = 0.15
    sigma: float = 0.017
    weight: float = 1.0
    betas: List[float] = field(default_factory=lambda: [1.0])


@dataclass
class Organism:
    """Decoded organism file fields used by Lenia.cpp:137-204."""
    cells: np.ndarray
    R: float = 13.0
    T: float = 10.0
    mu: float = 0.15
    sigma: float = 0.015


def _round_half_away(x: float) -> int:
    """std::round: halves round away from zero."""
    return int(math.copysign(math.floor(abs(float(x)) + 0.5), float(x)))


def _is_pow2(v: int) -> bool:
    return v != 0 and (v & (v - 1)) == 0


def _json_u32(v, default: int) -> int:
    """nlohmann value<uint32_t>: numbers truncate toward zero."""
    if v is None:
        return default
    return int(v) & 0xFFFFFFFF


class OracleLenia:
    """Restatement of LeniaModule (Modules/FieldModules/Lenia.cpp) on the CPU.

    ``params`` is the module's scene ``params`` object; ``organism`` supplies
    the decoded cells when ``params["organism"]`` names a file (the reference
    loads it from disk at setup, Lenia.cpp:300-313). ``precision`` is
    ``"ref32"`` or ``"f64"`` (module docstring). Two keys are extensions of
    this project and are read only here and in the product: ``kernelCore``
    (``"gaussShell"`` default, or ``"exp"``) and ``fftAnySize`` (default
    false = the reference's power-of-two rule, Lenia.cpp:245-251).
    """

    def __init__(self, params: dict, scene_w: int, scene_h: int, precision: str = "f64",
                 organism: Optional[Organism] = None, instance: str = "lenia0"):
        if precision not in ("ref32", "f64"):
            raise ValueError(precision)
        self.precision = precision
        self.instance = instance
        self.params = dict(params)
        self.warnings: List[str] = []
        self.base = {}
        for k, v in params.items():  # Scene.cpp:96-113
            if isinstance(v, bool):
                self.base[k] = 1.0 if v else 0.0
            elif isinstance(v, (int, float)):
                self.base[k] = _f32(v)
        self._setup(scene_w, scene_h, organism)
        self.seed_ = 0
        self.needs_init = True
        self.state = None
        self.init_override = None

    # Lenia.cpp:208-408
    def _setup(self, scene_w, scene_h, organism):
        p = self.params
        self.use_fft = p.get("convMode", "direct") == "fft"
        self.direct_multi = p.get("convMode", "direct") == "directMulti"
        self.core = CORE_EXP if p.get("kernelCore", "gaussShell") == "exp" else CORE_GAUSS_SHELL
        sw, sh = _json_u32(p.get("simWidth"), 0), _json_u32(p.get("simHeight"), 0)
        self.w = sw if sw else scene_w
        self.h = sh if sh else scene_h
        kj = p.get("kernels")
        has_kernels = isinstance(kj, list) and len(kj) > 0
        self.kernels: List[KernelDef] = []
        if has_kernels:
            for k in kj:
                if len(self.kernels) >= 4:
                    self.warnings.append("kernels truncated to 4")
                    break
                betas = [_f32(b) for b in k.get("betas", [])] or [1.0]
                self.kernels.append(KernelDef(_f32(k.get("radiusScale", 1.0)), _f32(k.get("mu", 0.15)),
                                              _f32(k.get("sigma", 0.017)), _f32(k.get("weight", 1.0)),
                                              betas))
        if self.use_fft and not p.get("fftAnySize", False) and not (
                _is_pow2(self.w) and _is_pow2(self.h)):
            self.warnings.append("fft requires power-of-two sim size; falling back to direct")
            self.use_fft = False
        multi = self.use_fft or self.direct_multi
        radius_scale_override = 1.0
        self.fallback_mu, self.fallback_sigma, self.fallback_dt = _f32(0.15), _f32(0.017), _f32(0.1)
        if has_kernels and not multi:
            self.warnings.append("kernels require convMode=fft; using kernels[0] in direct mode")
            k0 = self.kernels[0]
            radius_scale_override = k0.radius_scale
            self.fallback_mu, self.fallback_sigma = k0.mu, k0.sigma
        if not multi:
            self.kernels = []
        want_stamp = p.get("initMode", "noise") == "stamp"
        org_path = p.get("organism", "")
        want_org_params = bool(p.get("useOrganismParams", True))
        self.stamp_count = min(32, _json_u32(p.get("stampCount"), 6))
        self.stamp_rotate = bool(p.get("stampRotate", True))
        if org_path and want_org_params and has_kernels:
            want_org_params = False
        if want_stamp and not org_path:
            want_stamp = False
        org_radius_default = 13
        self.organism = organism if org_path else None
        if org_path and organism is None:
            want_stamp = False
        if self.organism is not None and want_org_params:
            org_radius_default = _round_half_away(np.float32(self.organism.R))
            self.fallback_mu = _f32(self.organism.mu)
            self.fallback_sigma = _f32(self.organism.sigma)
            if self.organism.T > 1e-6:
                self.fallback_dt = _f32(np.float32(1.0) / np.float32(self.organism.T))
        self.use_stamp = want_stamp and self.organism is not None
        r_json = _json_u32(p.get("radius"), org_radius_default)
        self.radius = _round_half_away(np.float32(r_json) * np.float32(radius_scale_override))
        self.init_coverage = _f32(p.get("initCoverage", 0.4))
        self.init_scale = _f32(p.get("initScale", 24.0))
        self.shell_mu = _f32(p.get("kernelShellMu", 0.5))
        self.shell_sigma = _f32(p.get("kernelShellSigma", 0.15))
        self.lut = direct_lut(self.radius, self.shell_mu, self.shell_sigma, self.core)

    def value(self, key: str, fallback: float, overrides: Optional[dict] = None) -> float:
        """SimulationModule::param -> ParameterBus::value with no mappings."""
        if overrides and key in overrides:
            return _f32(overrides[key])
        return self.base.get(key, _f32(fallback))

    def reset(self, seed: int) -> None:
        """Lenia.cpp:448-451."""
        self.seed_ = derive_seed(seed, LEN1_TAG)
        self.needs_init = True

    def set_initial_field(self, field_: np.ndarray) -> None:
        """The next init pass writes this field instead of noise/stamps."""
        self.init_override = np.ascontiguousarray(field_, np.float32).reshape(self.h, self.w)

    def _lo_params(self, fp: dict, seed: int, frame: int) -> LoParams:
        q = LoParams()
        q.dt, q.growth_mu, q.growth_sigma = fp["dt"], fp["growthMu"], fp["growthSigma"]
        q.noise_amount, q.mu_jitter, q.inject_amount = fp["noiseAmount"], fp["muJitter"], fp["injectAmount"]
        q.init_coverage, q.init_scale = self.init_coverage, self.init_scale
        q.inject_count, q.radius, q.kernel_size = fp["injectCount"], self.radius, 2 * self.radius + 1
        q.seed, q.width, q.height, q.frame_index, q.growth_mode = seed, self.w, self.h, frame, fp["growthMode"]
        return q

    def frame_params(self, overrides: Optional[dict] = None) -> dict:
        """Lenia.cpp:456-464."""
        v = lambda k, d: self.value(k, d, overrides)
        return {
            "dt": v("dt", self.fallback_dt), "growthMu": v("growthMu", self.fallback_mu),
            "growthSigma": v("growthSigma", self.fallback_sigma),
            "noiseAmount": v("noiseAmount", 0.0), "muJitter": v("muJitter", 0.0),
            "injectAmount": v("injectAmount", 0.0),
            "injectCount": int(np.float32(v("injectCount", 3.0)) + np.float32(0.5)),
            "growthMode": int(np.float32(v("growthMode", 1.0)) + np.float32(0.5)),
        }

    def _init(self, fp: dict, frame: int) -> None:
        """Lenia.cpp:468-558."""
        if self.init_override is not None:
            a = self.init_override.copy()
        elif self.use_stamp:
            a = np.zeros((self.h, self.w), np.float32)
            o = np.ascontiguousarray(self.organism.cells, np.float32)
            lib().lo_init_stamp(self.w, self.h, _ptr(o), o.shape[1], o.shape[0],
                                self.stamp_count, int(self.stamp_rotate), self.seed_, _ptr(a))
        else:
            a = np.zeros((self.h, self.w), np.float32)
            q = self._lo_params(fp, self.seed_, frame)
            lib().lo_init_noise(ctypes.byref(q), _ptr(a))
        self.state = a.astype(np.float64) if self.precision == "f64" else a
        if self.use_fft or self.direct_multi:
            eff = list(self.kernels) or [KernelDef(1.0, fp["growthMu"], fp["growthSigma"], 1.0, [1.0])]
            self.num_k = min(4, len(eff))
            self.kimg, self.kre, self.kim = [], [], []
            mp = LoMultiParams()
            for k in range(self.num_k):
                rk = _f32(np.float32(self.radius) * np.float32(eff[k].radius_scale))
                img = ring_image(self.w, self.h, rk, self.shell_sigma, eff[k].betas, self.core)
                self.kimg.append(img)
                if self.precision == "ref32" and self.use_fft:
                    re, im = fft2d_ref_f32(img, np.zeros_like(img), +1)
                    self.kre.append(re)
                    self.kim.append(im)
                mp.k_mu[k], mp.k_sigma[k], mp.k_weight[k] = eff[k].mu, eff[k].sigma, eff[k].weight
            for k in range(self.num_k, 4):
                mp.k_mu[k], mp.k_sigma[k], mp.k_weight[k] = 0.15, 0.017, 0.0
            mp.num_kernels = self.num_k
            self.multi = mp
        self.needs_init = False

    def potentials(self) -> List[np.ndarray]:
        """FP64 potentials u_k = K_k * A of the current state (multi-kernel)."""
        return [conv_circular_f64(self.state, k) for k in self.kimg]

    def encode(self, frame_index: int, substeps: int = 1, audio_frame: Optional[int] = None,
               overrides: Optional[dict] = None) -> np.ndarray:
        """Lenia.cpp:455-644. Returns the state after the frame's substeps."""
        fp = self.frame_params(overrides)
        if audio_frame is None:
            audio_frame = frame_index
        if self.needs_init:
            self._init(fp, frame_index)
        for s in range(max(1, substeps)):
            seed = pcg_hash(self.seed_ ^ ((frame_index * 197 + s) & 0xFFFFFFFF))
            self.step_once(fp, seed, frame_index, audio_frame)
        return self.state

    def step_once(self, fp: dict, seed: int, frame_index: int, audio_frame: int) -> None:
        """One substep with an explicit substep seed."""
        L = lib()
        if not (self.use_fft or self.direct_multi):
            q = self._lo_params(fp, seed, frame_index)
            dst = np.empty_like(self.state)
            lut = np.ascontiguousarray(self.lut)
            if self.precision == "ref32":
                L.lo_step_direct_f32(_ptr(self.state), _ptr(dst), _ptr(lut), ctypes.byref(q), audio_frame)
            else:
                L.lo_step_direct_f64(_ptr(self.state), _ptr(dst), _ptr(lut), ctypes.byref(q), audio_frame)
            self.state = dst
            return
        mp = self.multi
        mp.dt, mp.growth_mode = fp["dt"], fp["growthMode"]
        mp.noise_amount, mp.mu_jitter = fp["noiseAmount"], fp["muJitter"]
        mp.inject_amount, mp.inject_count = fp["injectAmount"], fp["injectCount"]
        mp.radius, mp.seed, mp.width, mp.height, mp.frame_index = self.radius, seed, self.w, self.h, frame_index
        dst = np.empty_like(self.state)
        if self.precision == "ref32" and self.use_fft:
            kre = np.ascontiguousarray(np.stack(self.kre))
            kim = np.ascontiguousarray(np.stack(self.kim))
            L.lo_step_fft_ref_f32(_ptr(self.state), _ptr(dst), _ptr(kre), _ptr(kim), ctypes.byref(mp), audio_frame)
        elif self.precision == "ref32":
            pots = [np.ascontiguousarray(conv_circular_f64(self.state, k).astype(np.float32)) for k in self.kimg]
            pots += [np.zeros_like(pots[0])] * (4 - len(pots))
            arr = (ctypes.c_void_p * 4)(*[p.ctypes.data for p in pots])
            L.lo_growth_multi_f32(_ptr(self.state), _ptr(dst), arr, ctypes.byref(mp), audio_frame)
        else:
            pots = [np.ascontiguousarray(p) for p in self.potentials()]
            pots += [np.zeros_like(pots[0])] * (4 - len(pots))
            arr = (ctypes.c_void_p * 4)(*[p.ctypes.data for p in pots])
            L.lo_growth_multi_f64(_ptr(self.state), _ptr(dst), arr, ctypes.byref(mp), audio_frame)
        self.state = dst


# ------------------------------------------------------- compiled reference

class RefEventIn(ctypes.Structure):
    _fields_ = [("type", ctypes.c_char * 32), ("curve", ctypes.c_char * 32), ("curve_value", ctypes.c_float),
                ("progress", ctypes.c_float), ("started", ctypes.c_int32), ("ended", ctypes.c_int32)]


class RefFeaturesIn(ctypes.Structure):
    """Per-frame inputs of the reference's bus (ref_shim/ref_runtime.cpp)."""
    _fields_ = [("env", (ctypes.c_float * 5) * 5), ("scalars", ctypes.c_float * 7), ("lanes", ctypes.c_float * 10),
                ("section_index", ctypes.c_int32), ("section_energy", ctypes.c_float),
                ("section_progress", ctypes.c_float), ("section_changed", ctypes.c_int32),
                ("section_role", ctypes.c_char * 32), ("num_events", ctypes.c_int32), ("events", RefEventIn * 4)]


REF_ENV_CHANNELS = ("kick", "snare", "hihat", "perc", "beat")
REF_ENV_PARTS = ("raw", "smoothed", "peak", "trigger", "hold")
REF_SCALARS = ("rms", "low", "mid", "high", "centroid", "flux", "time")
REF_LANES = ("tension", "intensity", "wet_ratio", "kick_gate", "macro_density", "macro_intensity",
             "master_rms", "drums_rms", "spatial_active", "se_env")


class RefBus:
    """The reference's ParameterBus (LifeCore/Params/ParameterBus.cpp), on its
    own or the bus of a RefLenia session."""

    def __init__(self, seed: int = 0, session: "Optional[RefLenia]" = None):
        L = RefLenia.lib()
        self._L = L
        self._own = session is None
        self.h_ = L.ref_bus_create(seed) if self._own else L.ref_session_bus(session.h_)
        self._session = session

    def __del__(self):
        if getattr(self, "_own", False) and getattr(self, "h_", None):
            self._L.ref_bus_destroy(self.h_)

    def load_scene(self, scene) -> None:
        err = ctypes.create_string_buffer(512)
        text = scene if isinstance(scene, str) else json.dumps(scene)
        if self._L.ref_bus_load_scene(self.h_, text.encode(), err, 512) != 0:
            raise ValueError(err.value.decode())

    def add_mapping(self, source, target, in_min=0.0, in_max=0.0, scale=1.0, offset=0.0, smoothing=0.0,
                    mode="add") -> None:
        if self._L.ref_bus_add_mapping(self.h_, source.encode(), target.encode(), in_min, in_max, scale, offset,
                                       smoothing, mode.encode()) != 0:
            raise ValueError(f"bad time source {source!r}")

    def set_base(self, key, v):
        self._L.ref_bus_set_base(self.h_, key.encode(), v)

    def set_override(self, key, v):
        self._L.ref_bus_set_override(self.h_, key.encode(), v)

    def clear_override(self, key):
        self._L.ref_bus_clear_override(self.h_, key.encode())

    def update(self, features: dict, dt: float, section_role: str = "", section_index: int = -1,
               events: Sequence[dict] = ()) -> None:
        """features: the names lenia_bus_set_feature takes ("kick.raw",
        "rms", "lane.tension", "section.energy", ...); events: dicts with
        type, progress, started, ended and optionally curve/curve_value."""
        f = RefFeaturesIn()
        for c, ch in enumerate(REF_ENV_CHANNELS):
            for p, part in enumerate(REF_ENV_PARTS):
                f.env[c][p] = features.get(f"{ch}.{part}", 0.0)
        for i, n in enumerate(REF_SCALARS):
            f.scalars[i] = features.get(n, 0.0)
        for i, n in enumerate(REF_LANES):
            f.lanes[i] = features.get("lane." + n, 0.0)
        f.section_index = section_index
        f.section_energy = features.get("section.energy", 0.0)
        f.section_progress = features.get("section.progress", 0.0)
        f.section_changed = int(features.get("section.changed", 0.0) != 0.0)
        f.section_role = section_role.encode()
        f.num_events = len(events)
        for i, e in enumerate(events):
            f.events[i].type = e["type"].encode()
            f.events[i].curve = e.get("curve", "").encode()
            f.events[i].curve_value = e.get("curve_value", 0.0)
            f.events[i].progress = e.get("progress", 0.0)
            f.events[i].started = int(e.get("started", False))
            f.events[i].ended = int(e.get("ended", False))
        self._L.ref_bus_update(self.h_, ctypes.byref(f), dt)

    def value(self, key, fallback=0.0) -> float:
        return self._L.ref_bus_value(self.h_, key.encode(), fallback)


class RefLenia:
    """The reference's own Lenia module + shaders compiled for the CPU."""

    _L = None

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(REF_SO)

    @classmethod
    def lib(cls):
        if cls._L is None:
            L = ctypes.CDLL(REF_SO)
            P, u32 = ctypes.c_void_p, ctypes.c_uint32
            L.ref_create.restype = P
            L.ref_create.argtypes = [ctypes.c_char_p, u32, u32, ctypes.c_char_p]
            L.ref_destroy.argtypes = [P]
            L.ref_set_base.argtypes = [P, ctypes.c_char_p, ctypes.c_float]
            L.ref_reset.argtypes = [P, u32]
            L.ref_set_init_field.argtypes = [P, P, ctypes.c_size_t]
            L.ref_encode.argtypes = [P, u32, u32, u32]
            L.ref_last_encode_seconds.restype = ctypes.c_double
            L.ref_last_encode_seconds.argtypes = [P]
            L.ref_field_size.argtypes = [P, ctypes.POINTER(u32), ctypes.POINTER(u32)]
            L.ref_get_field.argtypes = [P, P, ctypes.c_size_t]
            L.ref_put_field.argtypes = [P, P, ctypes.c_size_t]
            L.ref_get_upload.restype = ctypes.c_size_t
            L.ref_get_upload.argtypes = [P, ctypes.c_char_p, P, ctypes.c_size_t]
            L.ref_set_row_window.argtypes = [P, u32, u32]
            L.ref_pass_count.restype = ctypes.c_uint64
            L.ref_pass_count.argtypes = [P]
            L.ref_pcg.restype = u32
            L.ref_pcg.argtypes = [u32]
            L.ref_rand.restype = ctypes.c_float
            L.ref_rand.argtypes = [u32, u32, u32, u32]
            L.ref_bus_create.restype = P
            L.ref_bus_create.argtypes = [u32]
            L.ref_bus_destroy.argtypes = [P]
            L.ref_bus_load_scene.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]
            L.ref_bus_add_mapping.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_float,
                                              ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                              ctypes.c_char_p]
            L.ref_bus_set_base.argtypes = [P, ctypes.c_char_p, ctypes.c_float]
            L.ref_bus_set_override.argtypes = [P, ctypes.c_char_p, ctypes.c_float]
            L.ref_bus_clear_override.argtypes = [P, ctypes.c_char_p]
            L.ref_bus_update.argtypes = [P, ctypes.POINTER(RefFeaturesIn), ctypes.c_float]
            L.ref_bus_value.restype = ctypes.c_float
            L.ref_bus_value.argtypes = [P, ctypes.c_char_p, ctypes.c_float]
            L.ref_session_bus.restype = P
            L.ref_session_bus.argtypes = [P]
            L.ref_colormap.argtypes = [P, u32, u32, P, P, u32, u32]
            L.ref_npy_write.argtypes = [ctypes.c_char_p, P, ctypes.c_size_t, P, u32, ctypes.c_char_p,
                                        ctypes.c_size_t]
            L.ref_npy_read.argtypes = [ctypes.c_char_p, P, u32, P, ctypes.c_size_t, ctypes.c_char_p,
                                       ctypes.c_size_t]
            cls._L = L
        return cls._L

    def __init__(self, params: dict, scene_w: int, scene_h: int, instance: str = "lenia0"):
        L = self.lib()
        self.h_ = L.ref_create(json.dumps(params).encode(), scene_w, scene_h, instance.encode())
        if not self.h_:
            raise RuntimeError("reference module setup failed")
        w, h = ctypes.c_uint32(), ctypes.c_uint32()
        L.ref_field_size(self.h_, ctypes.byref(w), ctypes.byref(h))
        self.w, self.h = w.value, h.value
        self._init = None

    def __del__(self):
        if getattr(self, "h_", None) and self._L is not None:
            self._L.ref_destroy(self.h_)
            self.h_ = None

    def set_base(self, key: str, value: float) -> None:
        self.lib().ref_set_base(self.h_, key.encode(), value)

    def reset(self, seed: int) -> None:
        self.lib().ref_reset(self.h_, seed)

    def set_initial_field(self, f: Optional[np.ndarray]) -> None:
        if f is None:
            self.lib().ref_set_init_field(self.h_, None, 0)
            self._init = None
        else:
            self._init = np.ascontiguousarray(f, np.float32).ravel()
            self.lib().ref_set_init_field(self.h_, _ptr(self._init), self._init.size)

    def encode(self, frame_index: int, substeps: int = 1, audio_frame: Optional[int] = None) -> np.ndarray:
        if audio_frame is None:
            audio_frame = frame_index
        self.lib().ref_encode(self.h_, frame_index, substeps, audio_frame)
        return self.field()

    def last_encode_seconds(self) -> float:
        return float(self.lib().ref_last_encode_seconds(self.h_))

    def field(self) -> np.ndarray:
        out = np.empty(self.w * self.h, np.float32)
        rc = self.lib().ref_get_field(self.h_, _ptr(out), out.size)
        if rc != 0:
            raise RuntimeError("ref_get_field failed")
        return out.reshape(self.h, self.w)

    def put_field(self, f: np.ndarray) -> None:
        a = np.ascontiguousarray(f, np.float32).ravel()
        self.lib().ref_put_field(self.h_, _ptr(a), a.size)

    def upload(self, suffix: str) -> np.ndarray:
        n = self.lib().ref_get_upload(self.h_, suffix.encode(), None, 0)
        out = np.empty(n, np.float32)
        if n:
            self.lib().ref_get_upload(self.h_, suffix.encode(), _ptr(out), n)
        return out

    def set_row_window(self, y0: int, y1: int) -> None:
        """Only rows [y0, y1) of the update passes run (y1 = 0: all rows)."""
        self.lib().ref_set_row_window(self.h_, y0, y1)

    def pass_count(self) -> int:
        return int(self.lib().ref_pass_count(self.h_))


def ref_colormap(field: np.ndarray, cm: dict, out_w: int, out_h: int) -> np.ndarray:
    """The reference's colorMapField / colorMapFieldScaled (Shaders/Render/
    ColorMap.metal, compiled for the CPU) on a float32 field: out_h x out_w x
    4 floats, before the RGBA16F texture's rounding. cm: a, b, c, d (3 each),
    inputScale, inputBias, exposure, channel."""
    L = RefLenia.lib()
    f = np.ascontiguousarray(field, np.float32)
    h, w = f.shape
    p = np.array(list(cm["a"]) + list(cm["b"]) + list(cm["c"]) + list(cm["d"])
                 + [cm["inputScale"], cm["inputBias"], cm["exposure"]], np.float32)
    params = np.concatenate([p, np.array([cm["channel"]], np.uint32).view(np.float32)])
    out = np.empty((out_h, out_w, 4), np.float32)
    if L.ref_colormap(_ptr(f), w, h, _ptr(params), _ptr(out), out_w, out_h) != 0:
        raise RuntimeError("reference colour map kernel missing")
    return out


def ref_npy_write(path: str, a: np.ndarray) -> None:
    """The reference's writeNPYFloat32 (LifeCore/IO/NpyWriter.cpp)."""
    L = RefLenia.lib()
    a = np.ascontiguousarray(a, np.float32)
    shape = np.array(a.shape, np.uint32)
    err = ctypes.create_string_buffer(512)
    if L.ref_npy_write(os.fsencode(path), _ptr(a), a.size, _ptr(shape), a.ndim, err, 512) != 0:
        raise ValueError(err.value.decode())


def ref_npy_read(path: str, shape) -> np.ndarray:
    """The reference's readNPYFloat32 with an expected shape."""
    L = RefLenia.lib()
    shp = np.array(list(shape), np.uint32)
    out = np.empty(tuple(int(x) for x in shape), np.float32)
    err = ctypes.create_string_buffer(512)
    if L.ref_npy_read(os.fsencode(path), _ptr(shp), shp.size, _ptr(out), out.size, err, 512) != 0:
        raise ValueError(err.value.decode() or "read failed")
    return out
