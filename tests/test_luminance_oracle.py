"""The oracle's luminance_half (image.rs:401-428) with the flat-field mesh
(calibration.rs:362-379), checked on the CPU against a second, numpy float32
restatement of the same steps (every operation rounded to f32 in the
reference's order)."""
import ctypes as C

import numpy as np

F = np.float32


def _gain(gains, cols, rows, x, y, width, height):
    if cols < 2 or rows < 2:
        return F(1.0)
    cmax, rmax = F(cols - 1), F(rows - 1)
    fx = min(max(F(F(x / F(width)) * cmax), F(0.0)), cmax)
    fy = min(max(F(F(y / F(height)) * rmax), F(0.0)), rmax)
    c0, r0 = int(np.floor(fx)), int(np.floor(fy))
    c1, r1 = min(c0 + 1, cols - 1), min(r0 + 1, rows - 1)
    tx, ty = F(fx - F(c0)), F(fy - F(r0))
    g = lambda c, r: gains[r * cols + c]
    one = F(1.0)
    top = F(F(g(c0, r0) * F(one - tx)) + F(g(c1, r0) * tx))
    bottom = F(F(g(c0, r1) * F(one - tx)) + F(g(c1, r1) * tx))
    return F(F(top * F(one - ty)) + F(bottom * ty))


def _argument(samples, width, height, black, white, gains, cols, rows):
    w, h = width // 2, height // 2
    rng = max(F(F(white) - F(black)), F(1.0))
    out = np.zeros(w * h, np.float32)
    for j in range(h):
        for i in range(w):
            a, b = F(samples[2 * j, 2 * i]), F(samples[2 * j, 2 * i + 1])
            c, d = F(samples[2 * j + 1, 2 * i]), F(samples[2 * j + 1, 2 * i + 1])
            s = F(F(F(a + b) + c) + d)
            flat = _gain(gains, cols, rows, F(F(2.0) * F(i)) + F(0.5), F(F(2.0) * F(j)) + F(0.5), width, height)
            linear = F(max(F(F(F(s * F(0.25)) - F(black)) / rng), F(0.0)) * flat)
            out[j * w + i] = F(F(1.0) + F(F(1000.0) * linear))
    return out


def _oracle(lib, samples, width, height, black, white, gains, cols, rows):
    w, h = width // 2, height // 2
    out = np.zeros(w * h, np.float32)
    arg = np.zeros(w * h, np.float32)
    gp = gains.ctypes.data_as(C.POINTER(C.c_float)) if gains is not None else None
    lib.oracle_luminance_half_mesh(samples.ctypes.data_as(C.POINTER(C.c_uint16)), width, height, black, white, gp,
                                   cols, rows, out.ctypes.data_as(C.POINTER(C.c_float)),
                                   arg.ctypes.data_as(C.POINTER(C.c_float)))
    return out, arg


def test_oracle_argument_matches_float32_restatement(oracle_lib):
    rng = np.random.default_rng(11)
    for width, height, cols, rows in [(6, 4, 0, 0), (13, 9, 2, 2), (20, 14, 5, 4), (9, 7, 3, 6)]:
        samples = rng.integers(0, 65535, (height, width), dtype=np.uint16)
        gains = rng.uniform(0.7, 1.8, cols * rows).astype(np.float32) if cols else None
        black, white = float(F(rng.uniform(0, 4096))), float(F(rng.uniform(20000, 262080)))
        _, arg = _oracle(oracle_lib, samples, width, height, black, white, gains, cols, rows)
        expect = _argument(samples, width, height, black, white, gains, cols, rows)
        assert np.array_equal(arg.view(np.uint32), expect.view(np.uint32)), (width, height, cols, rows)


def test_oracle_flat_field_form_is_the_meshless_form(oracle_lib):
    rng = np.random.default_rng(3)
    samples = rng.integers(0, 65535, (30, 40), dtype=np.uint16)
    a, _ = _oracle(oracle_lib, samples, 40, 30, 4096.0, 262080.0, None, 0, 0)
    b = np.zeros(20 * 15, np.float32)
    oracle_lib.oracle_luminance_half(samples.ctypes.data_as(C.POINTER(C.c_uint16)), 40, 30, 4096.0, 262080.0,
                                     b.ctypes.data_as(C.POINTER(C.c_float)))
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
