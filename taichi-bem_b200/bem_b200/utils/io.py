"""[..., 1|2] real/complex packing (src/BEM_functions/utils/io.py:4-30)."""
import torch


def warp_tensor(x: torch.Tensor):
    n_ = x.shape[-1]
    if n_ == 1:
        return x.squeeze(-1)
    if n_ == 2:
        return torch.complex(x[..., 0], x[..., 1])
    raise NotImplementedError(
        f"warp_tensor: last dimension {n_} is neither 1 (real values) nor 2 (interleaved complex pairs)")


def unwarp_tensor(x: torch.Tensor):
    if x.is_complex():
        return torch.stack((x.real, x.imag), -1)
    return x.unsqueeze(-1)
