"""The CUDA library loads on a CPU-only host and exports every entry point
declared in include/profess_b200.h (no compute calls)."""
import os
import re

import pytest

from profess_b200 import build, native

HEADER = os.path.join(build.INCLUDE, "profess_b200.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ofdft_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_drop_in_entry_points():
    names = declared()
    for n in ("ofdft_calculate_potential_plus", "ofdft_proj_norm_rho_minimization", "ofdft_slot_create",
              "ofdft_engine_create", "ofdft_slot_forces", "ofdft_calculate_potential_plus_noalloc"):
        assert n in names


@pytest.mark.parametrize("which", ["cuda", "emu"])
def test_library_exports_every_declared_symbol(which):
    path = build.build_cuda() if which == "cuda" else build.build_emu()
    import ctypes
    lib = ctypes.CDLL(path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_header():
    names = set(declared())
    bound = set(native.SIGNATURES) | {"ofdft_last_error", "ofdft_calculate_potential_plus_noalloc"}
    assert names <= bound, sorted(names - bound)
