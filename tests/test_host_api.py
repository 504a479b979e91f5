"""Host-side API checks that need no GPU: constructor validation with the reference's
messages (sparse_sign.jl:71-127, count_sketch.jl:65-80, srht.jl:67-77, fjlt.jl FJLT
constructor, gaussian.jl:54-60, randsvd.jl:342-352, rangefinder.jl), the generic
fallbacks (src/Compressors.jl:146-153, :225-232, :338-359) and loud failure when no
device is present."""
import numpy as np
import pytest


def test_sparse_sign_checks(rla):
    with pytest.raises(rla.ArgumentError, match="Field `compression_dim` must be positive."):
        rla.SparseSign(compression_dim=0)
    with pytest.raises(rla.ArgumentError, match="Number of non-zero indices, 9, must be less than or equal to "
                                                 "compression dimension, 8."):
        rla.SparseSign(compression_dim=8, nnz=9)
    with pytest.raises(rla.ArgumentError, match="Field `nnz` must be positive."):
        rla.SparseSign(compression_dim=8, nnz=0)
    s = rla.SparseSign(compression_dim=10)
    assert s.nnz == 8 and s.cardinality == rla.Left() and s.type is np.float64
    assert rla.SparseSign(compression_dim=3).nnz == 3
    with pytest.raises(rla.ArgumentError, match="New `compression_dim`, 4, must be greater than or equal to "
                                                 "current `nnz`, 8."):
        s.compression_dim = 4
    with pytest.raises(rla.ArgumentError, match="New `nnz`, 11, must be less than or equal to current "
                                                 "`compression_dim`, 10."):
        s.nnz = 11
    s.nnz = 5
    assert s.nnz == 5


def test_other_constructors(rla):
    with pytest.raises(rla.ArgumentError, match="Field 'compression_dim' must be positive."):
        rla.CountSketch(compression_dim=0)
    with pytest.raises(rla.ArgumentError, match="`Undef\\(\\)` is not allowed"):
        rla.CountSketch(cardinality=rla.Undef())
    with pytest.raises(rla.ArgumentError, match="Field `block_size` must be positive."):
        rla.SRHT(block_size=0)
    with pytest.raises(rla.ArgumentError, match="Cardinality must be of type `Left` or `Right`."):
        rla.SRHT(cardinality=rla.Undef())
    with pytest.raises(rla.ArgumentError, match="Field `sparsity` must be between 0 and 1."):
        rla.FJLT(sparsity=1.5)
    with pytest.raises(rla.ArgumentError, match="Field 'compression_dim' must be positive."):
        rla.Gaussian(compression_dim=-1)
    with pytest.raises(rla.ArgumentError, match="Field `power_its` must be non-negative."):
        rla.RandSVD(power_its=-1)
    with pytest.raises(rla.ArgumentError, match="Field `block_size` must be non-negative."):
        rla.RandSVD(block_size=-1)
    with pytest.raises(rla.ArgumentError, match="Field `power_its` must be non-negative."):
        rla.RangeFinder(power_its=-2)
    r = rla.RandSVD()
    assert isinstance(r.compressor, rla.SparseSign) and r.compressor.cardinality == rla.Right()


def test_generic_fallbacks(rla):
    class MyCompressor(rla.Compressor):
        pass

    with pytest.raises(rla.ArgumentError, match="No `complete_compressor` method exists"):
        rla.complete_compressor(MyCompressor(), np.zeros((3, 3)))
    with pytest.raises(rla.ArgumentError, match="No method `update_compressor` exists"):
        rla.update_compressor_(object())
    with pytest.raises(rla.ArgumentError, match="No method `mul!` defined"):
        rla.mul_(np.zeros(2), np.zeros(2), np.zeros(2))

    class MyApprox(rla.Approximator):
        pass

    with pytest.raises(rla.ArgumentError, match="No method `complete_approximator` exists"):
        rla.complete_approximator(MyApprox(), np.zeros((3, 3)))


def test_no_device_fails_loudly(rla):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(rla.RLAError, match="no CPU fallback"):
        rla.complete_compressor(rla.SRHT(compression_dim=4), np.zeros((16, 2)))
