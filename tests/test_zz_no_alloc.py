"""adf_cpml_profiles_static: the CPML profiles with fixed device scratch.

Collected last on purpose: its first call performs the per-device scratch
set-up, and it must give the same results whether or not other GPU work ran
in the process before it.
"""
import numpy as np
import pytest

C0 = 343.0
DX = 0.005
DT = 0.7 * DX / (np.sqrt(3.0) * C0)

CASES = [(10, DT, 2000.0), (0, DT, 3000.0), (1, DT, 3000.0), (7, 2.309e-6, 10e3)]


@pytest.mark.gpu
def test_static_scratch_matches_allocating_entry(adf, ctx):
    # the largest size the fixed scratch takes, as the library reports it
    for npml, dt, fc in CASES + [(adf.static_cpml_max_npml(), DT, 2000.0)]:
        thick = DX * npml if npml else 0.0
        ref32, ref64 = adf.cpml_profiles(npml, C0, dt, 1e-4, thick, fc, ctx=ctx)
        # two calls in a row: the second reuses the scratch the first left behind
        for _ in range(2):
            o32, o64 = adf.cpml_profiles_static(npml, C0, dt, 1e-4, thick, fc, ctx=ctx)
            # same kernel, same inputs: bit for bit
            assert np.array_equal(o32, ref32), npml
            assert np.array_equal(o64, ref64), npml


@pytest.mark.gpu
def test_static_scratch_rejects_npml_beyond_its_size(adf, ctx):
    n = adf.static_cpml_max_npml() + 1
    with pytest.raises(RuntimeError, match="exceeds the fixed scratch"):
        adf.cpml_profiles_static(n, C0, DT, 1e-4, DX * n, 2000.0, ctx=ctx)
    # the context stays usable afterwards
    o32, _ = adf.cpml_profiles_static(10, C0, DT, 1e-4, DX * 10, 2000.0, ctx=ctx)
    r32, _ = adf.cpml_profiles(10, C0, DT, 1e-4, DX * 10, 2000.0, ctx=ctx)
    assert np.array_equal(o32, r32)
