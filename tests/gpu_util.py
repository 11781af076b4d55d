"""Helpers shared by the GPU parity tests: oracle grids wrapped as Raven-style grids."""

import types

import numpy as np

import oracle as O

LAWS = {
    # name: (oracle law, oracle form, oracle volume flux, product law factory, product form factory)
    "adv_weak": (O.LAW_ADVECTION, O.FORM_WEAK, O.FLUX_CENTRAL),
    "adv_fdc": (O.LAW_ADVECTION, O.FORM_FLUXDIFF, O.FLUX_CENTRAL),
    "eul_weak": (O.LAW_EULER, O.FORM_WEAK, O.FLUX_CENTRAL),
    "eul_fdc": (O.LAW_EULER, O.FORM_FLUXDIFF, O.FLUX_CENTRAL),
    "eul_kg": (O.LAW_EULER, O.FORM_FLUXDIFF, O.FLUX_KG),
    "eul_ec": (O.LAW_EULER, O.FORM_FLUXDIFF, O.FLUX_EC),
}


def product_scheme(rb, name, dim, adv=None):
    law_o, form_o, vf_o = LAWS[name]
    if law_o == O.LAW_ADVECTION:
        law = rb.AdvectionLaw(dim, adv)
    else:
        law = rb.EulerLaw(dim)
    vf = {O.FLUX_CENTRAL: rb.CentralFlux(), O.FLUX_KG: rb.KennedyGruberFlux(), O.FLUX_EC: rb.EntropyConservativeFlux()}[vf_o]
    form = rb.WeakForm() if form_o == O.FORM_WEAK else rb.FluxDifferencingForm(vf)
    return law, form


def oracle_law(name, dim, adv=None):
    law_o, form_o, vf_o = LAWS[name]
    return O.Law(law_o, dim, form=form_o, volume_flux=vf_o, adv=adv)


def wrap_oracle_grid(og):
    """A Raven-style grid object holding exactly the oracle's arrays."""
    r, w, D = og.lgl()
    cell = types.SimpleNamespace(dim=og.dim, nq=og.nq, r=r, w=w, D=D)
    g = types.SimpleNamespace(
        cell=cell, dim=og.dim, nq=og.nq, np=og.np, nfp=og.nfp, nfaces=og.nfaces, E=og.E,
        points=og.points(), volume_metrics=og.volume_metrics(), surface_metrics=og.surface_metrics(),
        vmapM=og.vmapM(), vmapP=og.vmapP(), boundarycodes=og.boundary(),
    )
    g.volume_weights = lambda: g.volume_metrics[:, g.dim * g.dim + 1, :]
    return g


def initial_state(og, olaw, name, seed=0, amp=0.05):
    """A smooth initial condition plus a seeded perturbation (keeps rho, p > 0)."""
    dim = og.dim
    if LAWS[name][0] == O.LAW_ADVECTION:
        q = og.initial_condition(olaw, 0)
    else:
        q = og.initial_condition(olaw, 1)
    rng = np.random.default_rng(seed)
    q = q * (1 + amp * rng.standard_normal(q.shape))
    return np.asfortranarray(q)


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
