"""The torch.library operators are registered and infer their output shapes
without running (fake tensors; no GPU needed)."""
import torch


def test_ops_registered_with_shapes():
    import pocketsdr_b200.ops  # noqa: F401  (registers the operators)
    from torch._subclasses.fake_tensor import FakeTensorMode
    with FakeTensorMode():
        buf = torch.empty(96000, dtype=torch.uint8, device="cuda")
        chips = torch.empty((5, 1023), dtype=torch.int8, device="cuda")
        grid, b, off, cn0, fd = torch.ops.pocketsdr.search(buf, 0, chips, [-500.0, 0.0, 500.0],
                                                           24e6, 4e6, 1e-3, 24000, 24000, 2)
        assert grid.shape == (5, 3, 24000) and grid.dtype == torch.float32
        assert b.shape == off.shape == cn0.shape == fd.shape == (5,)
        assert (b.dtype, off.dtype, cn0.dtype, fd.dtype) == (torch.int32, torch.int32,
                                                             torch.float32, torch.float64)
        banks = torch.empty((2, 10 * 24000, 2), dtype=torch.int8, device="cuda")
        c = torch.ops.pocketsdr.corr_batch(buf, [0, 7], [4e6, 4e6], [0.0, 0.1], [0.0, 3.5], banks,
                                           [0.0, -11.7, 11.7, -120.0], 24e6, 24000)
        assert c.shape == (2, 4) and c.dtype == torch.complex64


def test_torch_stream_names_the_legacy_stream(monkeypatch):
    """Torch's default stream (handle 0) goes to the C ABI as cudaStreamLegacy,
    since a NULL stream means the calling thread's own stream to some entry
    points; any other stream handle passes through."""
    from types import SimpleNamespace
    from pocketsdr_b200._lib import CUDA_STREAM_LEGACY, torch_stream
    for handle, want in ((0, CUDA_STREAM_LEGACY), (0x7F3A10, 0x7F3A10)):
        monkeypatch.setattr(torch.cuda, "current_stream",
                            lambda h=handle: SimpleNamespace(cuda_stream=h))
        assert torch_stream() == want
