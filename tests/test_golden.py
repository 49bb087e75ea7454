"""The committed golden fixtures (tests/golden, written by make_golden.py).

On the CPU, the oracle reproduces them bit for bit, so any change to the oracle
shows here. On the GPU, the CUDA stage reproduces them through the C ABI
without consulting the oracle at run time.
"""
import functools

import pytest

from golden import fixture


@pytest.mark.parametrize("name", fixture.NAMES)
def test_oracle_reproduces_golden(oracle_lib, name):
    g = fixture.load(name)
    got = fixture.run(g, oracle_lib.oracle_refine_multiview_depth, extra=(1,))
    fixture.compare(got, g)


@pytest.mark.gpu
@pytest.mark.parametrize("name", fixture.NAMES)
def test_gpu_stage_reproduces_golden(gpu_ctx, name):
    g = fixture.load(name)
    got = fixture.run(g, functools.partial(gpu_ctx.lib.chiaro_refine_multiview_depth, gpu_ctx.handle))
    fixture.compare(got, g)
