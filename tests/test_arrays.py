"""Argument checks of the Python entry points on the host (no GPU).  The
kernels index their arrays by one length on one device, so the checks refuse
anything else before a pointer reaches the library.  CUDA tensors are
stood in for by CPU tensors that report themselves as CUDA tensors on a
chosen device (the checks only read those attributes)."""
import pytest
import torch

from pfblob._arrays import Marshal, require


class FakeCuda(torch.Tensor):
    fake_device = torch.device("cuda", 0)

    @property
    def is_cuda(self):
        return True

    @property
    def device(self):
        return self.fake_device


def cuda_like(t, index=0):
    f = t.as_subclass(FakeCuda)
    f.fake_device = torch.device("cuda", index)
    return f


DEV0 = torch.device("cuda", 0)


def test_require_accepts_matching_tensors():
    a = cuda_like(torch.zeros(5, dtype=torch.float64))
    b = cuda_like(torch.ones(5, dtype=torch.float64))
    require(5, DEV0, x=a, y=b)
    require(5, DEV0, dtype=torch.int32, piv=cuda_like(torch.zeros(5, dtype=torch.int32)))


def test_require_refuses_host_tensors_and_arrays():
    import numpy as np
    with pytest.raises(TypeError, match="x must be a CUDA tensor"):
        require(3, DEV0, x=torch.zeros(3, dtype=torch.float64))
    with pytest.raises(TypeError, match="CUDA tensor"):
        require(3, DEV0, x=np.zeros(3))


def test_require_refuses_wrong_length_dtype_layout_and_device():
    with pytest.raises(ValueError, match="y has 4 elements, expected 5"):
        require(5, DEV0, x=cuda_like(torch.zeros(5, dtype=torch.float64)),
                y=cuda_like(torch.zeros(4, dtype=torch.float64)))
    with pytest.raises(TypeError, match="must be torch.float64"):
        require(5, DEV0, g=cuda_like(torch.zeros(5, dtype=torch.float32)))
    strided = cuda_like(torch.zeros(10, dtype=torch.float64))[::2]
    with pytest.raises(ValueError, match="contiguous"):
        require(5, DEV0, vx=strided)
    with pytest.raises(ValueError, match="is on cuda:1"):
        require(5, DEV0, vy=cuda_like(torch.zeros(5, dtype=torch.float64), index=1))


def test_marshal_refuses_arguments_on_two_devices():
    m = Marshal(device=0)
    m.dev(cuda_like(torch.zeros(3, dtype=torch.float64), 0), "xBlob")
    with pytest.raises(ValueError, match="yBlob is on cuda:1"):
        m.dev(cuda_like(torch.zeros(3, dtype=torch.float64), 1), "yBlob")


def test_marshal_follows_the_first_device_argument():
    m = Marshal(device=0)
    m.dev(cuda_like(torch.zeros(3, dtype=torch.float64), 1), "xBlob")
    assert m.device == torch.device("cuda", 1)
