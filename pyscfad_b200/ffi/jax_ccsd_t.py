"""JAX counterpart of pyscfad.cc.ccsd_t.kernel over the XLA FFI handlers.

Mirrors pyscfad/cc/ccsd_t.py:28-80: ``kernel(mycc, eris, t1, t2)`` is a
``jax.custom_vjp`` whose forward returns E(T) and whose backward returns
``(eris_bar, t1_bar, t2_bar)`` with nonzero ``fock`` (its [nocc:, :nocc]
block), ``mo_energy``, ``ovoo``, ``ovov`` and ``ovvv`` leaves and zeros for
every other leaf (:48-77).  Both directions run on this package's CUDA
kernels through ``ct_energy_ffi`` / ``ct_energy_vjp_ffi``
(pyscfad_b200/ffi/ct_xla_ffi.cc), which must have been built against jaxlib's
FFI headers and loaded with :func:`register`.

JAX is not a dependency of this package: importing this module without jax
raises ImportError, and nothing else imports it.
"""
from __future__ import annotations

import ctypes

import jax
import jax.numpy as jnp
from jax.tree_util import tree_flatten_with_path, tree_unflatten

MODES = {"fp64": 0, "tf32": 1, "bf16x3": 2}


def register(ffi_library_path: str) -> None:
    """Registers the two handlers of the built FFI library with XLA (CUDA)."""
    lib = ctypes.CDLL(ffi_library_path)
    for name in ("ct_energy_ffi", "ct_energy_vjp_ffi"):
        jax.ffi.register_ffi_target(name, jax.ffi.pycapsule(getattr(lib, name)), platform="CUDA")


def _layouts(eris, t1, t2):
    """Kernel layouts of pyscfad/cc/ccsd_t.py:88-106 (ovvv unpacked when packed)."""
    nocc, nvir = t1.shape
    ovvv = eris.get_ovvv() if hasattr(eris, "get_ovvv") else eris.ovvv
    vvop = jnp.concatenate([jnp.asarray(eris.ovov).transpose(1, 3, 0, 2),
                            jnp.asarray(ovvv).transpose(1, 3, 0, 2)], axis=3)
    return (jnp.asarray(eris.mo_energy), t1.T, t2.transpose(2, 3, 1, 0),
            jnp.asarray(eris.ovoo).transpose(1, 0, 3, 2), jnp.asarray(eris.fock)[nocc:, :nocc], vvop)


def _pack_tril(x):
    nvir = x.shape[-1]
    ii, jj = jnp.tril_indices(nvir)
    return x[..., ii, jj]


def kernel(mycc, eris, t1=None, t2=None, mode: str = "fp64"):
    t1 = mycc.t1 if t1 is None else t1
    t2 = mycc.t2 if t2 is None else t2
    m = MODES[mode]
    scalar = jax.ShapeDtypeStruct((), jnp.float64)

    @jax.custom_vjp
    def _ccsd_t_kernel(eris, t1, t2):
        args = _layouts(eris, t1, t2)
        return jax.ffi.ffi_call("ct_energy_ffi", scalar)(*args, mode=m)

    def _fwd(eris, t1, t2):
        return _ccsd_t_kernel(eris, t1, t2), (eris, t1, t2)

    def _bwd(res, ybar):
        eris, t1, t2 = res
        nocc, nvir = t1.shape
        args = _layouts(eris, t1, t2)
        outs = (scalar,) + tuple(jax.ShapeDtypeStruct(a.shape, jnp.float64) for a in args)
        _, mo_b, t1_b, t2_b, vooo_b, fvo_b, vvop_b = jax.ffi.ffi_call("ct_energy_vjp_ffi", outs)(
            *args, mode=m, et_bar=jnp.asarray(ybar, jnp.float64))
        # un-transpose (pyscfad/cc/ccsd_t.py:179-191); ovvv gradient symmetrised,
        # diagonal halved and tril-packed when eris.ovvv is stored packed
        nmo = nocc + nvir
        fock_bar = jnp.zeros((nmo, nmo)).at[nocc:, :nocc].set(fvo_b)
        ovvv_bar = vvop_b[:, :, :, nocc:].transpose(2, 0, 3, 1)
        if eris.ovvv.ndim == 3:
            ovvv_bar = ovvv_bar + ovvv_bar.transpose(0, 1, 3, 2)
            ovvv_bar = ovvv_bar.at[:, :, jnp.arange(nvir), jnp.arange(nvir)].multiply(0.5)
            ovvv_bar = _pack_tril(ovvv_bar)
        key_to_bar = {"fock": fock_bar, "mo_energy": mo_b, "ovoo": vooo_b.transpose(1, 0, 3, 2),
                      "ovov": vvop_b[:, :, :, :nocc].transpose(2, 0, 3, 1), "ovvv": ovvv_bar}
        path_vals, treedef = tree_flatten_with_path(eris)
        leaves = []
        for path, val in path_vals:
            name = path[0].name
            leaves.append(key_to_bar[name] if name in key_to_bar else jnp.zeros(jnp.shape(val)))
        return tree_unflatten(treedef, leaves), t1_b.T, t2_b.transpose(3, 2, 0, 1)

    _ccsd_t_kernel.defvjp(_fwd, _bwd)
    return _ccsd_t_kernel(eris, t1, t2)
