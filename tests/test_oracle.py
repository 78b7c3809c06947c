"""Pins the FP64 oracle (oracle/fft_oracle.c) against the reference crate's
own known-answer tests and against numpy's FFT.  CPU only."""
import math

import numpy as np
import pytest

from oracle import oracle as O


def test_length_four_forward_dft_known_answer():
    # src/math/mod.rs:575-612 (computes_known_length_four_forward_dft and the
    # f64 variant): [1,2,3,4] -> [10, -2+2i, -2, -2-2i], Normalization::None.
    x = np.array([1, 2, 3, 4], dtype=np.complex128)
    expected = np.array([10, -2 + 2j, -2, -2 - 2j])
    f64 = O.c2c_nd_f64(x, [4], normalization=O.NORM_NONE)
    assert np.max(np.abs(f64 - expected)) < 1e-12
    f32 = O.c2c_nd_dft_f32(x, [4], normalization=O.NORM_NONE)
    assert np.max(np.abs(f32 - expected)) < 1e-5


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 12, 16, 17, 30, 49, 97, 128, 210, 282, 1060,
                               1523, 3946])
@pytest.mark.parametrize("inverse", [False, True])
def test_fft_f64_matches_plain_dft(n, inverse):
    # src/math/mod.rs f64_fft_matches_a_plain_dft: input sin(0.37 i) + i cos(0.11 i),
    # agreement within 1e-12 of the largest component.
    i = np.arange(n)
    x = np.sin(i * 0.37) + 1j * np.cos(i * 0.11)
    sign = 1.0 if inverse else -1.0
    jk = np.outer(np.arange(n), np.arange(n)) % n
    W = np.exp(sign * 2j * np.pi * jk / n)
    expected = W @ x
    actual = O.fft_f64(x, inverse)
    scale = max(1.0, float(np.max(np.maximum(np.abs(expected.real), np.abs(expected.imag)))))
    assert np.max(np.maximum(np.abs(actual.real - expected.real),
                             np.abs(actual.imag - expected.imag))) < 1e-12 * scale


def test_batched_odd_axis_subset():
    # src/math/mod.rs f64_reference_computes_batched_odd_axis_subset.
    x = np.arange(1, 13, dtype=np.complex128)
    out = O.c2c_nd_f64(x, [2, 3], axes=[1], batch=2, normalization=O.NORM_NONE)
    root = math.sqrt(3.0) * 0.5
    exp = np.zeros(12, dtype=np.complex128)
    for b in range(2):
        base = b * 6
        for xx in range(2):
            a, bb, c = x[base + xx].real, x[base + 2 + xx].real, x[base + 4 + xx].real
            exp[base + xx] = a + bb + c
            exp[base + 2 + xx] = complex(a - 0.5 * (bb + c), root * (c - bb))
            exp[base + 4 + xx] = complex(a - 0.5 * (bb + c), root * (bb - c))
    assert np.max(np.abs(out - exp)) < 1e-12


def test_axis_subset_known_answer():
    # src/math/mod.rs computes_axis_subset_for_nd_shape: shape [2,3], axes [0].
    x = np.arange(1, 7, dtype=np.complex128)
    out = O.c2c_nd_dft_f32(x, [2, 3], axes=[0], normalization=O.NORM_NONE)
    assert np.max(np.abs(out - np.array([3, -1, 7, -1, 11, -1]))) < 1e-5


def test_packed_r2c_known_answer():
    # src/math/mod.rs computes_known_r2c_packed_even_length.
    out = O.r2c_packed_f64(np.array([1.0, 2.0, 3.0, 4.0]), [4], normalization=O.NORM_NONE)
    assert np.max(np.abs(out - np.array([10, -2 + 2j, -2]))) < 1e-12


def test_r2c_c2r_round_trip_odd_length():
    # src/math/mod.rs r2c_c2r_round_trip_odd_length.
    x = np.array([0.25, -1.0, 2.0, 0.5, -0.75])
    packed = O.r2c_packed_f64(x, [5], normalization=O.NORM_NONE)
    assert packed.size == 3
    back = O.c2r_from_packed_f64(packed, [5], normalization=O.NORM_INVERSE)
    assert np.max(np.abs(back - x)) < 1e-12


def test_r2c_c2r_round_trip_nd_packs_axis_zero():
    # src/math/mod.rs r2c_c2r_round_trip_nd_packs_axis_zero.
    x = np.array([0.25, -1.0, 2.0, 0.5, -0.75, 1.25])
    packed = O.r2c_packed_f64(x, [3, 2], normalization=O.NORM_NONE)
    assert packed.size == 4
    back = O.c2r_from_packed_f64(packed, [3, 2])
    assert np.max(np.abs(back - x)) < 1e-12


def test_inverse_default_normalization_recovers_input():
    # src/math/mod.rs inverse_default_normalization_recovers_input and the ND form.
    x = np.array([1 + 0.25j, 2 - 0.5j, -3 + 1j, 4 + 2j, 0.75 - 1.5j, -2.25 + 0.5j])
    spec = O.c2c_nd_f64(x, [2, 3], normalization=O.NORM_NONE)
    back = O.c2c_nd_f64(spec, [2, 3], inverse=True)
    assert np.max(np.abs(back - x)) < 1e-12


def test_pure_tone_maps_to_one_bin():
    # src/cpu.rs:1041-1079: a 256x128x8 complex exponential with
    # Normalization::Forward transforms to a unit delta (1e-9).
    shape = [256, 128, 8]
    k = (5, 17, 3)
    i0 = np.arange(256)[None, None, :]
    i1 = np.arange(128)[None, :, None]
    i2 = np.arange(8)[:, None, None]
    ph = 2 * np.pi * (k[0] * i0 / 256 + k[1] * i1 / 128 + k[2] * i2 / 8)
    x = np.exp(1j * ph).reshape(-1)
    out = O.c2c_nd_f64(x, shape, normalization=O.NORM_FORWARD)
    peak = (k[2] * 128 + k[1]) * 256 + k[0]
    exp = np.zeros_like(out)
    exp[peak] = 1.0
    assert np.max(np.abs(out - exp)) < 1e-9


@pytest.mark.parametrize("shape,axes,batch", [([16], None, 3), ([6, 10], None, 2),
                                              ([5, 7, 9], [2, 0], 1), ([127], None, 2),
                                              ([1009], None, 1), ([4099], None, 1)])
def test_oracle_matches_numpy(shape, axes, batch):
    rng = np.random.default_rng(7)
    n = int(np.prod(shape)) * batch
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    out = O.c2c_nd_f64(x, shape, axes=axes, batch=batch, normalization=O.NORM_NONE)
    arr = x.reshape([batch] + shape[::-1])
    ax = list(range(len(shape))) if axes is None else axes
    np_axes = [len(shape) - a for a in ax]
    ref = np.fft.fftn(arr, axes=np_axes).reshape(-1)
    assert O.rel_l2(out, ref) < 1e-14


def test_rader_permutation_and_primitive_roots():
    # src/runtime/rader_axis.rs:2852 rader_permutation_covers_nonzero_prime_indices;
    # smallest primitive roots (src/runtime/axis_policy.rs:134-152).
    perm = O.rader_permutation(17)
    assert sorted(perm.tolist()) == list(range(1, 17))
    g = O.primitive_root(17)
    assert g == 3
    assert perm.tolist() == [pow(g, k + 1, 17) for k in range(16)]
    assert O.primitive_root(1009) == 11
    assert O.primitive_root(4099) == 2
    assert O.primitive_root(7) == 3


def test_factorisation_matches_reference_order():
    # src/runtime/mod.rs:30-57: greedy 13, 11, 8, 7, 5, 4, 3, 2.
    assert O.factor_supported_length(1024) == [8, 8, 8, 2]
    assert O.factor_supported_length(15015) == [13, 11, 7, 5, 3]
    assert O.factor_supported_length(17) is None
    assert O.factor_supported_length(21) == [7, 3]


def test_df64_split_join_round_trip():
    # src/math/double_float.rs:22-33: hi = f32(x), lo = f32(x - hi).
    v = np.array([1.0 / 3.0 + 1j * math.pi, -2.0 ** -30 + 1e-12j])
    w = O.df64_split(v)
    assert w.dtype == np.float32 and w.size == 8
    assert w[0] == np.float32(1.0 / 3.0)
    back = O.df64_join(w)
    assert np.max(np.abs(back - v) / np.abs(v)) < 2.0 ** -44


def test_chirp_square_reduced_modulo_2n():
    # src/runtime/bluestein_axis.rs:1806-1818: n = 1_000_003, i = 999_999 gives
    # i^2 mod 2n = 1_000_019.
    n, i = 1_000_003, 999_999
    assert (i * i) % (2 * n) == 1_000_019


def test_cpu_baseline_plan_matches_oracle():
    rng = np.random.default_rng(3)
    for shape in ([1024], [6, 10], [17], [34]):
        n = int(np.prod(shape)) * 2
        x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
        ref = O.c2c_nd_f64(x.astype(np.complex128), shape, batch=2)
        y = x.copy()
        O.cpu_c2c_f32_inplace(y, shape, batch=2)
        assert O.rel_l2(y, ref) < 2e-6
