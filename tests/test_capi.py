"""The C ABI library on the CPU: it loads, exports every entry point that
include/lenia_b200.h declares, and its host logic (parameter parsing and
the reference's setup fallbacks) resolves like the reference. No compute
call needs a device here."""
import ctypes
import json
import os
import re
import subprocess

import pytest

import life_simulation_b200 as lb
from tests.conftest import GOLDEN, ROOT, reference_preset

HEADER = os.path.join(ROOT, "include", "lenia_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lenia_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lb.load_library()
    out = subprocess.run(["nm", "-D", "--defined-only", lb.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (lenia_\w+)", out))
    decl = declared_functions()
    assert decl, "no declarations parsed"
    missing = [f for f in decl if f not in exported]
    assert not missing, missing
    assert set(decl) == set(lb.EXPORTS)


def test_header_compiles_as_c():
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-x", "c", HEADER],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_status_strings():
    L = lb.load_library()
    assert L.lenia_status_string(0) == b"ok"
    assert b"CUDA" in L.lenia_status_string(-3)


def preset(name):
    return reference_preset(name.replace(".json", ""))[0]


def test_inspect_direct_default():
    r = lb.inspect({"radius": 13}, 256, 256)
    assert r["conv_mode"] == lb.CONV_DIRECT and r["radius"] == 13 and r["status"] == 0


def test_inspect_fft_pow2_rule_falls_back_like_reference():
    p = {"convMode": "fft", "simWidth": 1920, "simHeight": 1080, "radius": 24,
         "kernels": [{"betas": [1.0], "radiusScale": 0.5}]}
    r = lb.inspect(p, 1280, 720)
    assert r["status"] == lb.LENIA_WARN_FALLBACK
    assert r["conv_mode"] == lb.CONV_DIRECT
    assert r["radius"] == 12  # round(24 * kernels[0].radiusScale)
    assert "powers of two" in r["warning"] and "kernels[0]" in r["warning"]


def test_inspect_fft_any_size_mixed_radix():
    p = {"convMode": "fft", "fftAnySize": True, "simWidth": 1920, "simHeight": 1080, "radius": 24,
         "kernels": [{"betas": [1.0]}] * 3}
    r = lb.inspect(p, 1920, 1080)
    assert r["status"] == 0 and r["conv_mode"] == lb.CONV_FFT and r["num_kernels"] == 3
    prod = lambda xs: eval("*".join(map(str, xs)))
    assert prod(r["fft_radix_row"]) == 960 and prod(r["fft_radix_col"]) == 1080


def test_inspect_unsupported_fft_size_falls_back():
    p = {"convMode": "fft", "fftAnySize": True, "simWidth": 98, "simHeight": 70, "radius": 5}
    r = lb.inspect(p, 98, 70)  # 49 = 7^2 has no 2/3/5 plan
    assert r["conv_mode"] == lb.CONV_DIRECT and r["status"] == lb.LENIA_WARN_FALLBACK


def test_inspect_kernels_truncated_to_four():
    p = {"convMode": "fft", "simWidth": 64, "simHeight": 64, "kernels": [{"betas": [1.0]}] * 6}
    r = lb.inspect(p, 64, 64)
    assert r["num_kernels"] == 4 and "truncating" in r["warning"]


def test_inspect_stamp_without_organism_falls_back():
    r = lb.inspect({"initMode": "stamp"}, 64, 64)
    assert r["use_stamp_init"] == 0 and "organism" in r["warning"]


def test_inspect_organism_params(tmp_path):
    org = tmp_path / "o.json"
    org.write_text(json.dumps({"R": 11.5, "T": 4, "mu": 0.2, "sigma": 0.03, "cells": [[0.5, 1.0], [0.0, 0.25]]}))
    r = lb.inspect({"initMode": "stamp", "organism": str(org)}, 64, 64)
    assert r["use_stamp_init"] == 1 and r["radius"] == 12 and r["status"] == 0
    bad = tmp_path / "bad.json"
    bad.write_text(json.dumps({"cells": [[0.5, 1.5]]}))
    r = lb.inspect({"initMode": "stamp", "organism": str(bad)}, 64, 64)
    assert r["use_stamp_init"] == 0 and "out of [0,1]" in r["warning"]


def test_inspect_reference_presets():
    r = lb.inspect(preset("lenia_multikernel.json"), 1280, 720)
    assert (r["sim_width"], r["sim_height"], r["conv_mode"], r["num_kernels"], r["radius"]) == (
        1024, 512, lb.CONV_FFT, 3, 24)
    r = lb.inspect(preset("lenia_basic.json"), 768, 768)
    assert (r["conv_mode"], r["radius"]) == (lb.CONV_DIRECT, 13)
    r = lb.inspect(preset("lenia_orbium.json"), 1280, 720, base_dir=GOLDEN)
    assert r["use_stamp_init"] == 1 and r["radius"] == 13


def test_inspect_bad_json():
    with pytest.raises(lb.LeniaError):
        lb.inspect("{not json", 64, 64)


_CTYPES = {"uint32_t": ctypes.c_uint32, "int32_t": ctypes.c_int32, "int": ctypes.c_int, "size_t": ctypes.c_size_t,
           "float": ctypes.c_float, "double": ctypes.c_double, "uint64_t": ctypes.c_uint64}


def declared_signatures():
    """(return type, name, [parameter types]) of every declaration."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = []
    for ret, name, args in re.findall(r"^\s*((?:const\s+)?\w+\s*\**)\s*(lenia_\w+)\s*\(([^;]*?)\)\s*;", text,
                                      flags=re.S | re.M):
        params = [] if args.strip() in ("", "void") else [" ".join(a.split()) for a in args.split(",")]
        types = [p.rsplit(" ", 1)[0] if "*" not in p else "ptr" for p in params]
        out.append((" ".join(ret.split()), name, types))
    return out


def test_every_entry_point_rejects_null_arguments():
    # Null handles and null pointers (zero sizes) come back as
    # LENIA_ERR_INVALID_ARG before any device work; the message getters
    # return a string for a null handle. A separate handle on the library
    # keeps these argtypes apart from the package's.
    L = ctypes.CDLL(lb.LIB_PATH)
    sigs = declared_signatures()
    assert {n for _, n, _ in sigs} == set(declared_functions())
    checked = 0
    for ret, name, types in sigs:
        fn = getattr(L, name)
        fn.argtypes = [ctypes.c_void_p if t == "ptr" else _CTYPES[t.replace("const ", "")] for t in types]
        args = [None if t == "ptr" else 0 for t in types]
        if ret == "int":
            fn.restype = ctypes.c_int
            assert fn(*args) == -1, name  # LENIA_ERR_INVALID_ARG
            checked += 1
        elif ret == "const char*" and name != "lenia_status_string":
            fn.restype = ctypes.c_char_p
            assert isinstance(fn(*args), bytes), name
    assert checked >= 60


def test_inspect_reports_the_direct_radius_limit_like_setup():
    # The direct path holds R <= 32 (per kernel for directMulti); inspection
    # (setup's host half) rejects what setup would, the spectral path not.
    with pytest.raises(lb.LeniaError, match="status -2"):
        lb.inspect({"radius": 40}, 256, 256)
    assert lb.inspect({"radius": 32}, 256, 256)["status"] == 0
    two = [{"radiusScale": 1.0}, {"radiusScale": 2.0}]
    with pytest.raises(lb.LeniaError, match="kernel radius <= 32"):
        lb.inspect({"radius": 20, "convMode": "directMulti", "kernels": two}, 256, 256)
    assert lb.inspect({"radius": 16, "convMode": "directMulti", "kernels": two}, 256, 256)["radius"] == 16
    assert lb.inspect({"radius": 40, "convMode": "fft"}, 256, 256)["conv_mode"] == lb.CONV_FFT
    # A non-power-of-two size falls back to direct, where R = 40 is refused.
    with pytest.raises(lb.LeniaError, match="radius <= 32"):
        lb.inspect({"radius": 40, "convMode": "fft"}, 250, 256)


_ALLOC_FAILURE_CHILD = r"""
import ctypes, resource, sys
sys.path.insert(0, sys.argv[1])
import life_simulation_b200 as lb
L = lb.load_library()
cfg = lb.config_from_params({"convMode": "fft", "radius": 9})
fp = lb.make_frame_params(growth_sigma=0.02)
# Cap the address space a little above what the process maps now, so the
# call's host tables (a twiddle table of width/2 entries: 1 GiB here) cannot
# be allocated.
soft, hard = resource.getrlimit(resource.RLIMIT_AS)
used = int(open("/proc/self/statm").read().split()[0]) * resource.getpagesize()
resource.setrlimit(resource.RLIMIT_AS, (used + (256 << 20), hard))
w, h = 1 << 28, 1
# Aligned, distinct, never dereferenced on the host (the call fails before
# any device work).
rc = L.lenia_fft_step_noalloc(ctypes.c_void_p(1 << 20), ctypes.c_void_p(2 << 20), w, h, ctypes.byref(cfg),
                              ctypes.byref(fp), 1, None)
print(rc, L.lenia_noalloc_last_message().decode())
"""


def test_host_allocation_failure_is_a_status_not_an_exception():
    # A C++ std::bad_alloc inside an entry point must come back as a status
    # code with a message, never unwind through the C ABI (which would
    # abort the process). The child process caps its address space so the
    # entry point's host tables cannot be allocated.
    r = subprocess.run([os.sys.executable, "-c", _ALLOC_FAILURE_CHILD, ROOT], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    rc, msg = r.stdout.strip().split(" ", 1)
    assert int(rc) == -3 and "host allocation failed" in msg, r.stdout
