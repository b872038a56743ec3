"""torch.autograd binding of the effective-stiffness solve and its adjoint.

    model = EffectiveStiffness(phis, precision="mixed", rtol=1e-6)   # gray volumes [z, y, x]
    C = model(E)             # E: (B, Lz, Ly, Lx) float32 tensor with requires_grad -> (B, 6, 6) float64
    loss = ((C - C_target) ** 2).sum()
    loss.backward()          # E.grad from dtc_energy_grad (no second solve)

Forward: one dtc_solve_batch with the per-voxel moduli E (keep_displacements = 1; batches
larger than the device memory are solved in chunks whose displacements are checkpointed to
the host).  A CUDA tensor E on the solver's device goes through the device-pointer entries:
dtc_solve_batch_device_moduli reads it, dtc_energy_grad_device writes E.grad in place.  Backward: dL/dE_v = a * sum_{a,b} G_ab u_a,v^T Khat u_b,v with
G = vv^-1 dL/dff, the derivative of the energy products u_a^T K u_b of the converged load
cases -- the operator is self-adjoint, so the forward displacements are the adjoint solution.
The reference has no gradient; this is an extension of its homogenisation
(f-src/mod_struct_calcmat.f90:216-500) to differentiable moduli.
"""
import numpy as np
import torch

from . import Domain, Solver, synth


class _EffectiveStiffnessFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, E, module):
        on_device = E.is_cuda and E.device.index == module.device
        if on_device:
            # the moduli stay on the device: the library copies them once through its own pinned
            # buffer (dtc_solve_batch_device_moduli)
            e_dev = E.detach().to(torch.float32).contiguous()
            torch.cuda.current_stream(E.device).synchronize()
            doms = [Domain(p, E=module.E_ref, nu=module.nu, delta=module.delta, llimit=module.llimit)
                    for p in module.phis]
            res = module.solver.solve_device_moduli(doms, [e_dev[i].data_ptr() for i in range(e_dev.shape[0])])
        else:
            e_np = E.detach().to(torch.float32).cpu().numpy()
            doms = [Domain(p, E=module.E_ref, nu=module.nu, delta=module.delta,
                           E_voxel=np.ascontiguousarray(e_np[i]), llimit=module.llimit)
                    for i, p in enumerate(module.phis)]
            res = module.solver.solve(doms)
        ctx.on_device = on_device
        module._generation += 1
        ctx.module = module
        ctx.generation = module._generation
        ctx.shape = tuple(E.shape)
        ctx.device, ctx.dtype = E.device, E.dtype
        module.last = res
        C = np.stack([r["c"] for r in res])
        return torch.from_numpy(C).to(device=E.device)

    @staticmethod
    def backward(ctx, grad_c):
        m = ctx.module
        if m._generation != ctx.generation:
            raise RuntimeError("EffectiveStiffness: backward must follow its own forward (the solver keeps the "
                               "displacements of its last forward only)")
        dl = grad_c.detach().to(torch.float64).cpu().numpy()   # B x 36 values
        if ctx.on_device:
            g = torch.empty(ctx.shape, dtype=torch.float32, device=ctx.device)
            torch.cuda.current_stream(ctx.device).synchronize()
            m.solver.energy_grad_device(dl, [g[i].data_ptr() for i in range(ctx.shape[0])])
            return g.to(dtype=ctx.dtype), None
        grads = [np.zeros(ctx.shape[1:], np.float32) for _ in range(ctx.shape[0])]
        m.solver.energy_grad(dl, grads)
        g = torch.from_numpy(np.stack(grads)).to(device=ctx.device, dtype=ctx.dtype)
        return g, None


class EffectiveStiffness(torch.nn.Module):
    """C(E) for a fixed batch of gray volumes (the mesh, i.e. which voxels are bone, is fixed
    by the gray values and llimit; E only scales the kept voxels)."""

    def __init__(self, phis, *, delta=synth.DELTA, nu=synth.NU, E_ref=synth.E_CONST, llimit=1, precision="mixed",
                 rtol=1e-6, inner_precond="mg", estimator="energy", device=0, max_it=500000):
        super().__init__()
        self.phis = [np.asarray(p) for p in phis]
        self.delta, self.nu, self.E_ref, self.llimit = delta, nu, E_ref, llimit
        self.device = device
        self.solver = Solver(precision=precision, rtol=rtol, max_it=max_it, rotation_search=False, device=device,
                             keep_displacements=True, inner_precond=inner_precond, estimator=estimator)
        self._generation = 0
        self.last = None

    def forward(self, E):
        if E.dim() != 4 or E.shape[0] != len(self.phis):
            raise ValueError("E must be (B, Lz, Ly, Lx) with B = number of volumes")
        return _EffectiveStiffnessFn.apply(E, self)

    def close(self):
        self.solver.close()
