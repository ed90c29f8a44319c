"""Device integral engine (rijk_int2c2e_dev / rijk_int3c2e_dev) and the
all-device tensor build (rijk_build_rimatr_from_shells) against the host
engine, whose energies are pinned to REST's in test_scf_oracle.py.

Integrals agree with the host engine to 1e-12 of the largest element (both
evaluate the same McMurchie-Davidson expressions in FP64; only the summation
order differs).  The fitted tensors agree to 1e-10 of the largest element and
the SCF energies to 1e-9 Eh.
"""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

from rest_b200._abi import RijkError
from rest_b200.basis import Molecule, int2c2e, int2c2e_dev, int3c2e, int3c2e_dev
from rest_b200.scf import SCF, ScfOptions, metric_inv_sqrt
from rest_b200.scf_batch import water_cluster

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
TIGHT = dict(scf_acc_etot=1e-11, scf_acc_rho=1e-8, scf_acc_eev=1e-8, max_scf_cycle=200)


def _water():
    g = json.loads((GOLDEN / "water_rihf.json").read_text())
    return g, Molecule.from_angstrom(g["symbols"], g["coords_angstrom"])


def _molecule(name):
    if name == "water":
        return _water()[1]
    return water_cluster(3, seed=7)


@pytest.mark.parametrize("name", ["water", "cluster3"])
@pytest.mark.parametrize("auxbas", ["def2-SVP-JKFIT", "def2-SV(P)-JKFIT"])
def test_int2c2e_dev_matches_host(name, auxbas):
    aux = _molecule(name).shells(auxbas)
    ref = int2c2e(aux)
    got = int2c2e_dev(aux).cpu().numpy()
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", ["water", "cluster3"])
@pytest.mark.parametrize("basis", ["def2-SVP", "STO-3G"])
def test_int3c2e_dev_matches_host(name, basis):
    mol = _molecule(name)
    bas, aux = mol.shells(basis), mol.shells("def2-SVP-JKFIT")
    ref = int3c2e(bas, aux)  # (npair, naux)
    got = int3c2e_dev(bas, aux).cpu().numpy().T
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_build_from_shells_cholesky_matches_host_path(ctx):
    mol = water_cluster(3, seed=7)
    bas, aux = mol.shells("def2-SVP"), mol.shells("def2-SVP-JKFIT")
    ctx.build_rimatr_cholesky(int2c2e(aux), int3c2e(bas, aux), bas.nfun)
    ref = ctx.get_rimatr()
    ctx.build_rimatr_from_shells(bas, aux)
    got = ctx.get_rimatr()
    assert (ctx.num_basis, ctx.num_auxbas) == (bas.nfun, aux.nfun)
    assert np.max(np.abs(got - ref)) <= 1e-10 * np.max(np.abs(ref))


def test_build_from_shells_inv_sqrt_matches_host_path(ctx):
    mol = water_cluster(3, seed=7)
    bas, aux = mol.shells("def2-SVP"), mol.shells("def2-SVP-JKFIT")
    v2 = int2c2e(aux)
    factor = metric_inv_sqrt(v2)
    ctx.fit_rimatr(factor, int3c2e(bas, aux), bas.nfun)
    ref = ctx.get_rimatr()
    ctx.build_rimatr_from_shells(bas, aux, factor)
    got = ctx.get_rimatr()
    assert np.max(np.abs(got - ref)) <= 1e-10 * np.max(np.abs(ref))


@pytest.mark.parametrize("metric", ["inv_sqrt", "cholesky"])
def test_scf_with_device_integrals_matches_oracle(ctx, metric):
    g, mol = _water()
    r = SCF(mol, g["basis"], g["auxbas"], ScfOptions(metric=metric, integrals="device", **TIGHT), ctx=ctx).run()
    assert r.converged
    assert abs(r.energy - g["oracle_energy"]) < 1e-9


def test_device_engine_rejects_high_angular_momentum(ctx):
    """An AO set with g shells is beyond the device engine: refused before any launch."""
    mol = _water()[1]
    aux = mol.shells("def2-SVP-JKFIT")
    with pytest.raises(RijkError) as e:
        int3c2e_dev(aux, aux)
    assert e.value.status == 8  # RIJK_ERR_TOO_LARGE
    with pytest.raises(RijkError) as e:
        ctx.build_rimatr_from_shells(aux, aux)
    assert e.value.status == 8
    # the context still works afterwards
    bas = mol.shells("def2-SVP")
    ctx.build_rimatr_from_shells(bas, aux)
    assert ctx.num_basis == bas.nfun
    torch.cuda.synchronize()


@pytest.mark.parametrize("name", ["water", "cluster3"])
@pytest.mark.parametrize("basis", ["def2-SVP", "STO-3G"])
def test_nuclear_attraction_from_point_charges_matches_host(name, basis):
    """Nuclear attraction through the device three-centre engine, each nucleus an
    s Gaussian of exponent 1e20 (a point charge to double precision)."""
    from rest_b200.basis import int1e, int1e_nuclear_dev

    mol = _molecule(name)
    bas = mol.shells(basis)
    ref = int1e(mol, bas, "nuclear")
    got = int1e_nuclear_dev(mol, bas).cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
