"""Host-side caches of Hamiltonians and their device state: identity, not object ids."""

from __future__ import annotations

import gc

import pyticc_b200 as tb
from pyticc_b200 import scattering, workloads
from pyticc_b200.propagation import runner


def _system(mu_amu: float):
    return tb.build_ScattSystem(tb.AtomSpec(), workloads.rigid_rotor(20.0, 2), Jtot=1, system_parity=1, potential=workloads.lj_aniso_pes(150.0, 6.5, 0.3, 0.2), reduced_mass=mu_amu * tb.AMU2AU)


def test_a_new_system_is_never_served_a_collected_systems_hamiltonian():
    grid = tb.prepare_potential(_system(18.0), (3.0, 4.0), (0.1,), n_theta=6)
    for k in range(12):
        mu = 10.0 + k
        system = _system(mu)
        ham = scattering.hamiltonian_for(system, grid)
        assert ham.reduced_mass == mu * tb.AMU2AU
        assert scattering.hamiltonian_for(system, grid) is ham
        del system, ham
        gc.collect()


def test_the_hamiltonian_cache_is_bounded_and_holds_its_keys():
    grid = tb.prepare_potential(_system(18.0), (3.0, 4.0), (0.1,), n_theta=6)
    systems = [_system(5.0 + k) for k in range(scattering.HAMILTONIAN_CACHE_SIZE + 3)]
    hams = [scattering.hamiltonian_for(s, grid) for s in systems]
    assert len(scattering._HAMILTONIANS) <= scattering.HAMILTONIAN_CACHE_SIZE
    assert all(entry[1] is grid and entry[2].reduced_mass == entry[0].reduced_mass for entry in scattering._HAMILTONIANS.values())
    # the most recent ones are served from the cache, the oldest were rebuilt on demand
    assert scattering.hamiltonian_for(systems[-1], grid) is hams[-1]
    assert scattering.hamiltonian_for(systems[0], grid) is not hams[0]


def test_device_state_lives_on_its_hamiltonian():
    grid = tb.prepare_potential(_system(18.0), (3.0, 4.0), (0.1,), n_theta=6)
    a = scattering.hamiltonian_for(_system(7.0), grid)
    b = scattering.hamiltonian_for(_system(8.0), grid)
    built = []
    state_a = runner._device_state(a, ("probe",), lambda: built.append("a") or "A")
    state_b = runner._device_state(b, ("probe",), lambda: built.append("b") or "B")
    assert (state_a, state_b) == ("A", "B")
    assert runner._device_state(a, ("probe",), lambda: "other") == "A"
    runner.release_device_state(a)
    assert runner._device_state(a, ("probe",), lambda: "rebuilt") == "rebuilt"
    assert built == ["a", "b"]
    assert runner._device_state(object(), ("probe",), lambda: "uncached") == "uncached"
