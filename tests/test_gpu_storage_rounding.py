"""Stochastic rounding of the reduced storages on the GPU (hl_round_to_storage).

The stream-collide kernels store float16 / bfloat16 moments through one codec: a value goes to
one of its two representable neighbours, the upper one with probability equal to its distance
from the lower one in units of their spacing, the random bits a hash of the value, the cell and
the moment. hl_round_to_storage runs that codec on given values, so these tests check it
directly: every result is one of the two neighbours; over many cells the share rounded up
matches the distance (unbiased, normal and float16-subnormal values alike); the two-cell form
the TMA kernel uses gives the single form's results bit for bit; the result is a deterministic
function of value and place; non-finite values stay non-finite.
"""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

_DT = {"float16": (1, torch.float16, torch.int16), "bfloat16": (2, torch.bfloat16, torch.int16),
       "float32": (0, torch.float32, torch.int32), "float64": (3, torch.float64, torch.int64)}


def _round(values: torch.Tensor, storage: str, first_cell=0, paired=False) -> torch.Tensor:
    """values [n_moments, n_cells] float32 on the GPU -> the stored tensor"""
    from openhomelbm_b200 import _lib

    code, dt, _ = _DT[storage]
    nm, n = values.shape
    out = torch.empty((nm, n), dtype=dt, device=values.device)
    _lib.check(_lib.lib().hl_round_to_storage(values.data_ptr(), n, nm, code, first_cell, int(paired),
                                              out.data_ptr(), _lib.stream_ptr()), "round to storage")
    return out


def _neighbours(v: float, dt: torch.dtype):
    """the representable neighbours lo <= |v| <= hi of |v| in dt, as float64"""
    a = abs(v)
    rn = torch.tensor([a], dtype=torch.float64).to(torch.float32).to(dt)
    bits = int(rn.view(torch.int16).item())
    r = float(rn.double().item())
    if r == a:
        return r, r
    step = torch.tensor([bits - 1 if r > a else bits + 1], dtype=torch.int16).view(dt).double().item()
    return (step, r) if r > a else (r, step)


VALUES = [1.0 + 1.2345e-4, -3.3333e-2, 0.7, 1234.567, 6.0e-5, -2.5e-6, 3.0e-8, -4.4e-7, 6.10349998e-05, 1e-9,
          -0.5, 0.0]


@pytest.mark.parametrize("storage", ["float16", "bfloat16"])
def test_rounding_is_unbiased_and_lands_on_a_neighbour(storage):
    dt = _DT[storage][1]
    n = 1 << 17
    for v in VALUES:
        v32 = float(np.float32(v))
        x = torch.full((1, n), v32, dtype=torch.float32, device="cuda")
        got = _round(x, storage, first_cell=12345).double().cpu().numpy()[0]
        lo, hi = _neighbours(v32, dt)
        mag = np.abs(got)
        assert np.all((mag == lo) | (mag == hi)), (storage, v, np.unique(got)[:6])
        assert np.all((np.sign(got) == np.sign(v32)) | (got == 0)), (storage, v)
        if hi == lo:
            continue
        p = (abs(v32) - lo) / (hi - lo)
        up = float(np.mean(mag == hi))
        # 13 (float16) or 16 (bfloat16) random bits: the probability is the distance cut to
        # that many bits, a bias below 2^-13 of the spacing
        tol = 5.0 * math.sqrt(p * (1 - p) / n) + 2.0 ** -13 + 1.0 / n
        assert abs(up - p) <= tol, (storage, v, up, p, tol)


@pytest.mark.parametrize("storage", ["float16", "bfloat16", "float32"])
def test_two_cell_form_equals_single_form_and_is_deterministic(storage):
    g = torch.Generator(device="cpu").manual_seed(5)
    n = 1001  # odd: the last cell takes the single form in the paired call too
    x = (torch.rand((10, n), generator=g, dtype=torch.float64) - 0.5)
    scale = torch.pow(10.0, torch.randint(-9, 3, (10, n), generator=g).double())
    x = (x * scale).float().cuda()
    a = _round(x, storage, first_cell=777)
    b = _round(x, storage, first_cell=777, paired=True)
    c = _round(x, storage, first_cell=777)
    assert torch.equal(a.view(_DT[storage][2]), b.view(_DT[storage][2]))
    assert torch.equal(a.view(_DT[storage][2]), c.view(_DT[storage][2]))
    d = _round(x, storage, first_cell=778)  # another place, another rounding for some values
    if storage != "float32":
        assert not torch.equal(a.view(_DT[storage][2]), d.view(_DT[storage][2]))
    else:
        assert torch.equal(a, x)


@pytest.mark.parametrize("storage", ["float16", "bfloat16"])
def test_non_finite_values_stay_non_finite(storage):
    big = 7.0e4 if storage == "float16" else 3.4e38
    x = torch.tensor([[float("inf"), float("-inf"), float("nan"), big, -big, 1.0]], device="cuda")
    x = x.expand(64, 6).t().contiguous().view(1, -1)  # every value in 64 cells
    got = _round(x, storage).float().cpu().view(6, 64)
    assert torch.isposinf(got[0]).all() and torch.isneginf(got[1]).all() and torch.isnan(got[2]).all()
    top = torch.finfo(_DT[storage][1]).max  # beyond the largest finite value: it, or an infinity
    assert ((got[3] == top) | torch.isposinf(got[3])).all() and ((got[4] == -top) | torch.isneginf(got[4])).all()
    assert (got[5] == 1.0).all()


def test_float64_widens():
    x = torch.tensor([[0.1, -2.5e-30, 3.0]], dtype=torch.float32, device="cuda")
    assert torch.equal(_round(x, "float64"), x.double())
