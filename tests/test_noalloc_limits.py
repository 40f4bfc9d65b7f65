"""Limits of the allocation-free evaluation, checked on the host (no GPU).

ofdft_calculate_potential_plus_noalloc plans a call (slot descriptor, FFT
plans, task lists, scratch layout) on the host before its first CUDA call,
and refuses with OFDFT_EINVAL a request its fixed scratch cannot hold.  These
tests call it in a child process that sees no GPU (CUDA_VISIBLE_DEVICES
empty), with dummy addresses that are never dereferenced: a refused request
returns OFDFT_EINVAL, and a request the planner accepts gets as far as
looking for a device and returns OFDFT_ECUDA.  The sweep covers every
7-smooth grid with axes of 2 to 128 points and at most 262144 points, in both
WT forms (alpha = beta, three spectra; alpha != beta, four spectra), so
neither the task-list bound nor the scratch-size check is reached inside the
documented range."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes, json, sys
sys.path.insert(0, sys.argv[1])
from profess_b200 import native
lib = native.load_library()
fn = lib.ofdft_calculate_potential_plus_noalloc
fn.argtypes = [ctypes.POINTER(native.CellDesc), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
               ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
fn.restype = ctypes.c_int
lat = (ctypes.c_double * 9)(20, 0, 0, 0, 21, 0, 0, 0, 22)

def call(n, kinetic=4, alpha=5 / 6, beta=5 / 6, precision=native.FP64):
    d = native.CellDesc(n[0], n[1], n[2], lat, kinetic, 1.0, 1.0, alpha, beta, 2.7, 0.0, 0.0, 0.0, precision)
    # dummy non-null addresses: the call returns before it could use them
    rc = fn(ctypes.byref(d), 16, 16, 16, 1, 16, None, None)
    return rc, lib.ofdft_last_error().decode()

def smooth(m):
    for p in (2, 3, 5, 7):
        while m % p == 0:
            m //= p
    return m == 1

out = {"refused": {}, "accepted_bad": []}
for name, args in {"axis_129": ((129, 16, 16),), "axis_11": ((11, 16, 16),), "axis_256": ((256, 16, 16),),
                   "axis_1": ((1, 16, 16),), "points_over": ((128, 128, 32),),
                   "wgc": ((16, 16, 16), 5), "fp32": ((16, 16, 16), 4, 5 / 6, 5 / 6, native.FP32)}.items():
    out["refused"][name] = call(*args)
sizes = [m for m in range(2, 129) if smooth(m)]
count = 0
for a in sizes:
    for b in sizes:
        if a * b * 2 > 262144:
            continue
        for c in sizes:
            if a * b * c > 262144:
                continue
            for ab in ((5 / 6, 5 / 6), (1.2, 0.45)):
                rc, msg = call((a, b, c), 4, *ab)
                count += 1
                if rc != 2:  # OFDFT_ECUDA: planned, then no device
                    out["accepted_bad"].append([a, b, c, ab[0], rc, msg])
out["count"] = count
print(json.dumps(out))
"""


def _run_child():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-c", CHILD, ROOT], capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_noalloc_limits_on_the_host():
    from profess_b200 import build
    build.build_cuda()
    res = _run_child()
    for name, (rc, msg) in res["refused"].items():
        assert rc == 1, (name, rc, msg)  # OFDFT_EINVAL before any CUDA call
    assert "7-smooth" in res["refused"]["axis_129"][1] and "7-smooth" in res["refused"]["axis_11"][1]
    assert "262144" in res["refused"]["points_over"][1]
    assert res["count"] > 10000
    assert res["accepted_bad"] == []
