"""Diagonal preconditioners estimated from batched Jacobian products
(reference: diagonal_preconditioner_spatial / diagonal_preconditioner_fourier,
jax_scripts/lib/preconditioners.py:225-360).

Hutchinson's estimator diag(J) ~ mean_z z * (J z): each of the k rounds is one
batched JVP of `batch` probe vectors at the cached linearisation (one sweep of
the batched tangent kernels), where the reference vmaps its JVP.  The probes
are drawn with numpy's PCG64 seeded by `seed` where the reference splits a
jax.random key, so the estimate is statistically, not bitwise, the
reference's.

The Jacobian maps [T, fields, sx] to [pt, fields, px]; the reference
multiplies its probes (fields only) with the whole flattened output, whose
length differs by the two phase conditions.  Here the estimate is taken over
the fields block of the output, and the returned M divides the fields block of
its argument (a flat [T, fields, sx] vector or a fields tensor) and leaves T
and sx unchanged.
"""

from __future__ import annotations

import numpy as np
import torch


def _rademacher(rng, shape):
    """+-1 with probability 1/2 (preconditioners.py:232-234)."""
    return 2.0 * (rng.random(shape) < 0.5).astype(np.float64) - 1.0


def _jac_fields(input_dict, jac, z_fields):
    """Fields block of J [0, z, 0] for a batch of probes z [batch, 2, n, n]."""
    batch = z_fields.shape[0]
    dev = z_fields.device
    tan = {"fields": z_fields, "T": torch.zeros(batch, dtype=torch.float64, device=dev),
           "sx": torch.zeros(batch, dtype=torch.float64, device=dev)}
    return jac(input_dict, tan)["fields"]


def _divide_fields(diag):
    def M(v, mode=None):
        """v / diag on the fields block; the matrix is diagonal, so mode
        ("trans" / "no_trans") is ignored (preconditioners.py:268-288, :355-359); the estimate is not written
        to a .mat file as the reference does (:266, :350)."""
        if v.dim() == 1 and v.numel() == diag.numel() + 2:
            out = v.clone()
            out[1:-1] = v[1:-1] / diag.reshape(-1)
            return out
        return v / diag.reshape(v.shape)
    return M


def diagonal_estimate_spatial(input_dict, jac, k=8, batch=4, seed=0):
    """Real-space diagonal of the fields block of J, [2, n, n] (preconditioners.py:225-263)."""
    fields = input_dict["fields"]
    shape = tuple(fields.shape[-3:])
    nf = int(np.prod(shape))
    rng = np.random.default_rng(seed)
    diag = torch.zeros(nf, dtype=torch.float64, device=fields.device)
    for _ in range(k):                                                # :243
        z = torch.as_tensor(_rademacher(rng, (batch, nf)), device=fields.device)   # :249
        Jz = _jac_fields(input_dict, jac, z.reshape((batch,) + shape)).reshape(batch, nf)
        diag += torch.sum(z * Jz, dim=0)                              # :258
    return (diag / k / batch).reshape(shape)                          # :263


def diagonal_estimate_fourier(input_dict, jac, k=8, batch=4, seed=0):
    """The same estimate in the rfft2 basis with unit-modulus random phases,
    returned in real space, [2, n, n] (preconditioners.py:291-348)."""
    fields = input_dict["fields"]
    shape = tuple(fields.shape[-3:])
    n = shape[-1]
    rng = np.random.default_rng(seed)
    dev = fields.device
    diag = 0
    for _ in range(k):                                                # :323
        g = torch.as_tensor(rng.standard_normal((batch,) + shape), device=dev)
        z = torch.fft.rfft2(g)                                        # :306-311
        z = z / torch.abs(z)
        z_real = torch.fft.irfft2(z, s=(n, n))                        # :328-329
        Jz = torch.fft.rfft2(_jac_fields(input_dict, jac, z_real.contiguous()))   # :336-338
        diag = diag + torch.sum(torch.conj(z) * Jz, dim=0)            # :339
    diag = diag / k / batch                                           # :345
    return torch.fft.irfft2(diag, s=(n, n))                           # :348


def diagonal_preconditioner_spatial(input_dict, param_dict, jac, k=8, batch=4, seed=0):
    """M(v, mode) = v / diag with the spatial estimate (preconditioners.py:225-288)."""
    return _divide_fields(diagonal_estimate_spatial(input_dict, jac, k, batch, seed))


def diagonal_preconditioner_fourier(input_dict, jac, k=8, batch=4, seed=0):
    """M(v, mode) = v / diag with the Fourier-basis estimate (preconditioners.py:291-360)."""
    return _divide_fields(diagonal_estimate_fourier(input_dict, jac, k, batch, seed))
