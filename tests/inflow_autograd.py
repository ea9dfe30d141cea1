"""Thin test harness: the adjoint as a torch.autograd.Function.

theta (16 values) sets the inflow profile on the x = 0 face,
    u(j, k) = 1 + sum_{a,b<4} theta[4a+b] sin((a+1) pi y') sin((b+1) pi z'),
    y' = j / (ny - 1), z' = k / (nz - 1),
of an AdiSolver3D; the forward runs n_steps steps and returns the kinetic energy J
of a box, and backward maps the library's node-value gradient (adi_adjoint_run) to
theta through the same basis."""
import numpy as np
import torch


def inflow_basis(ny: int, nz: int, n: int = 4) -> np.ndarray:
    """[n*n, ny, nz] sine products, zero on the walls."""
    y = np.arange(ny) / (ny - 1)
    z = np.arange(nz) / (nz - 1)
    out = np.zeros((n * n, ny, nz))
    for a in range(n):
        for b in range(n):
            out[a * n + b] = np.outer(np.sin((a + 1) * np.pi * y), np.sin((b + 1) * np.pi * z))
    return out


def inflow_values(domain, theta: np.ndarray, base_u: float = 1.0):
    """The domain's node values with the inflow face interior set by theta."""
    vx = domain.vx.copy()
    phi = inflow_basis(domain.ny, domain.nz, int(round(np.sqrt(len(theta)))))
    prof = base_u + np.tensordot(np.asarray(theta, np.float64), phi, axes=1)
    vx[0, 1:-1, 1:-1] = prof[1:-1, 1:-1]
    return vx, domain.vy, domain.vz, domain.T


class InflowEnergy(torch.autograd.Function):
    """J(theta) with its adjoint gradient.  ctx keeps dJ/dtheta from the one
    forward + backward run the library does."""

    @staticmethod
    def forward(ctx, theta, solver, domain, init_state, run):
        th = theta.detach().cpu().numpy().astype(np.float64)
        solver.set_node_values(*inflow_values(domain, th))
        solver.set_state(*init_state)
        J, gnv, _ = solver.adjoint_run(*run)
        phi = inflow_basis(domain.ny, domain.nz, int(round(np.sqrt(len(th)))))
        g = np.tensordot(phi[:, 1:-1, 1:-1], gnv[0][0, 1:-1, 1:-1].astype(np.float64), axes=([1, 2], [0, 1]))
        ctx.save_for_backward(torch.as_tensor(g, dtype=theta.dtype))
        return theta.new_tensor(J)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None, None, None, None
