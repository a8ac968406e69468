"""Argument handling of the kernelFunctions_fort drop-in, without a GPU: f2py's
shape checks raise ValueError before any device work."""
import numpy as np
import pytest

from registration_b200 import kernelFunctions_fort as kff


def test_module_exports_the_f2py_routines():
    for nm in ("applyk", "applykdifft", "applykmat", "applykdiffmat", "applykdiff1", "applykdiff2",
               "applykdiff1and2", "applykdiff11", "applykdiff12", "applykdiff11and12"):
        assert callable(getattr(kff, nm))


@pytest.mark.parametrize("call", [
    lambda: kff.applyk(np.zeros((4, 3)), np.zeros((5, 3)), np.zeros((5, 2)), 0.1, 10, 3, 5, 3, 2),
    lambda: kff.applyk(np.zeros((4, 3)), np.zeros((5, 3)), np.zeros((6, 2)), 0.1, 10),
    lambda: kff.applyk(np.zeros((4, 3)), np.zeros((5, 2)), np.zeros((5, 2)), 0.1, 10),
    lambda: kff.applykdifft(np.zeros((4, 3)), np.zeros((5, 3)), np.zeros((1, 4, 3)), np.zeros((1, 5, 3)), 0.1, 10,
                            4, 5, 3, 3, 2),
    lambda: kff.applykdifft(np.zeros((4, 3)), np.zeros((5, 3)), np.zeros((1, 5, 3)), np.zeros((1, 5, 3)), 0.1, 10),
    lambda: kff.applykmat(np.zeros((4, 3)), np.zeros((5, 3)), np.zeros((4, 4, 1)), 0.1, 10),
    lambda: kff.applykdiffmat(np.zeros((4, 3)), np.zeros((5, 3)), np.zeros((5, 4)), 0.1, 10),
    lambda: kff.applykdiff1(np.zeros((4, 3)), np.zeros((4, 3)), np.zeros((3, 3)), 0.1, 10),
    lambda: kff.applykdiff11and12(np.zeros((4, 3)), np.zeros((4, 3)), np.zeros((4, 3)), np.zeros((4, 3)), 0.1, 10,
                                  4, 2),
    lambda: kff.applyk(np.zeros(4), np.zeros((5, 3)), np.zeros((5, 2)), 0.1, 10),
])
def test_shape_disagreements_raise_value_error(call):
    with pytest.raises(ValueError):
        call()


def test_precision_switch():
    assert kff.get_precision() == "fp32c"
    kff.set_precision("fp64")
    assert kff.get_precision() == "fp64"
    kff.set_precision("fp32c")
    with pytest.raises(ValueError):
        kff.set_precision("fp16")
