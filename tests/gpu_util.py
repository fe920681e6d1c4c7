"""Helpers for the GPU parity tests: host<->device moves and the comparison
rules (bit-exact integers/keys/permutations; f64 sums and means within
1e-12 relative, with the condition-aware bound |gpu - exact| <= 1e-12 *
sum|x| reported alongside for cancelling sums)."""
import numpy as np
import torch

F64_REL = 1e-12


def dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy()


def bits_equal(a: np.ndarray, b: np.ndarray) -> bool:
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype.itemsize == b.dtype.itemsize and \
        (a.view(f"u{a.dtype.itemsize}") == b.view(f"u{b.dtype.itemsize}")).all()


def assert_f64_close(got: np.ndarray, exact: np.ndarray, abs_sum: np.ndarray, what: str):
    """Both the plain relative check and the condition-aware one; fails if
    the condition-aware bound fails, and returns how many groups only passed
    the condition-aware bound (cancelling sums)."""
    got = np.asarray(got, np.float64)
    exact = np.asarray(exact, np.float64)
    err = np.abs(got - exact)
    cond_ok = err <= F64_REL * np.maximum(abs_sum, np.abs(exact)) + 1e-300
    assert cond_ok.all(), f"{what}: {np.count_nonzero(~cond_ok)} groups beyond 1e-12 * sum|x|, " \
                          f"worst {err[~cond_ok][:5]} vs {exact[~cond_ok][:5]}"
    rel_ok = err <= F64_REL * np.abs(exact)
    plain = int(np.count_nonzero(~rel_ok))
    print(f"{what}: {got.size} groups within 1e-12 * sum|x|; plain-relative failures: {plain}")
    return plain
