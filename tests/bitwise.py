"""Exact comparison for the parity tests.

Integer arrays must be equal. Floating arrays must hold equal values, with
equal signs of zero and NaN in the same places; NaN payloads are not
compared (the host's libm and the GPU produce different quiet-NaN bit
patterns for the same invalid operation)."""
import numpy as np


def assert_same(got, want, err_msg=""):
    got, want = np.asarray(got), np.asarray(want)
    np.testing.assert_array_equal(got, want, err_msg=err_msg)
    if got.dtype.kind == "f" or want.dtype.kind == "f":
        g, w = np.broadcast_arrays(got, want)
        both = ~(np.isnan(g) | np.isnan(w))
        np.testing.assert_array_equal(np.signbit(g[both]), np.signbit(w[both]),
                                      err_msg=err_msg or "signs of zero differ")
