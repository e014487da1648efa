"""ASE calculator on the B200 engine (gfn1-rs ``python/gfn1_rs/ase.py:115-434``).

``GFN1RSCalculator`` keeps the reference class's name, constructor keywords of
the plain path, result keys and unit rules: energies in eV (the free energy
``total_free``), forces in eV/Angstrom, Mulliken charges in e and the dipole in
e*Angstrom, with the native atomic-unit values beside them under ``native_*``
keys.  ``ase.units`` (Hartree, Bohr) is the single source of the conversion
factors when ASE is installed; without ASE the class still works on any object
with ``get_atomic_numbers``, ``get_positions`` and ``get_pbc`` and uses ASE's
default (CODATA 2014) values of the same two constants.

Beyond the reference: ``calculate_many`` evaluates a list of structures in one
batched engine call, and ``learned_guess=True`` starts each SCC from the
learned initial guess.  Periodic cells and the spectroscopy / response methods
of the reference class are outside the engine and raise ``ValueError``.
"""
from __future__ import annotations

from typing import Any

import numpy as np

from .native import Gfn1NativeCalculator

try:  # pragma: no cover - depends on the environment
    from ase.calculators.calculator import Calculator as _AseCalculator
    from ase.calculators.calculator import all_changes
    from ase.units import Bohr as _BOHR
    from ase.units import Hartree as _HARTREE
    from ase.units import invcm as _INVCM_EV
    HAVE_ASE = True
except ImportError:
    HAVE_ASE = False
    _HARTREE = 27.211386024367243  # ase.units.Hartree (CODATA 2014, ASE's default)
    _BOHR = 0.5291772105638411     # ase.units.Bohr (CODATA 2014)
    _INVCM_EV = 1.239841973964072e-04  # ase.units.invcm, eV per cm^-1 (CODATA 2014)
    all_changes = ("positions", "numbers", "cell", "pbc", "initial_charges", "initial_magmoms")

    class _AseCalculator:  # minimal stand-in with ASE's calculate/results protocol
        implemented_properties: list = []
        default_parameters: dict = {}

        def __init__(self, restart=None, label=None, atoms=None, **kwargs):
            self.parameters = dict(self.default_parameters)
            self.parameters.update(kwargs)
            self.results: dict = {}
            self.atoms = None
            self._last_key = None

        def set(self, **kwargs):
            changed = {k: v for k, v in kwargs.items() if self.parameters.get(k) != v}
            self.parameters.update(kwargs)
            if changed:
                self.results = {}
            return changed

        def calculate(self, atoms=None, properties=("energy",), system_changes=all_changes):
            if atoms is not None:
                self.atoms = atoms

        def get_property(self, name, atoms=None, allow_calculation=True):
            atoms = self.atoms if atoms is None else atoms
            key = (tuple(np.asarray(atoms.get_atomic_numbers()).tolist()),
                   np.asarray(atoms.get_positions(), dtype=float).tobytes())
            if key != self._last_key or name not in self.results:
                self.results = {}
                self.calculate(atoms, [name])
                self._last_key = key
            return self.results[name]

        def get_potential_energy(self, atoms=None, force_consistent=False):
            return self.get_property("energy", atoms)

        def get_forces(self, atoms=None):
            return self.get_property("forces", atoms)

        def get_charges(self, atoms=None):
            return self.get_property("charges", atoms)

        def get_dipole_moment(self, atoms=None):
            return self.get_property("dipole", atoms)

_ENERGY = _HARTREE
_FORCE = _HARTREE / _BOHR
_DIPOLE = _BOHR


class GFN1RSCalculator(_AseCalculator):
    """ASE calculator for non-periodic GFN1-xTB energy, forces, charges and dipole."""

    implemented_properties = ["energy", "forces", "charges", "dipole"]
    default_parameters = {
        "param_path": None,
        "charge": 0.0,
        "multiplicity": None,
        "level_shift": 0.0,
        "max_scc": 250,
        "energy_tolerance": 1.0e-6,
        "charge_tolerance": 2.0e-5,
        "mixing": 0.4,
        "scc_broyden": True,
        "scc_broyden_size": 250,
        "electronic_temperature": 300.0,
        "enable_dispersion": True,
        "learned_guess": False,
        "device": 0,
    }

    def __init__(self, restart: str | None = None, label: str | None = None, atoms=None, **kwargs: Any) -> None:
        _AseCalculator.__init__(self, restart=restart, label=label, atoms=atoms, **kwargs)
        self._native = None
        self._batch = None

    def set(self, **kwargs: Any):
        changed = _AseCalculator.set(self, **kwargs)
        if changed:
            self._native = None
            self._batch = None
        return changed

    def _options(self) -> dict:
        p = self.parameters
        return dict(max_scc=p["max_scc"], energy_tolerance=p["energy_tolerance"],
                    charge_tolerance=p["charge_tolerance"], mixing=p["mixing"], scc_broyden=p["scc_broyden"],
                    scc_broyden_size=p["scc_broyden_size"], electronic_temperature=p["electronic_temperature"],
                    enable_dispersion=p["enable_dispersion"])

    def _batch_calc(self):
        if self._batch is None:
            from .batch import BatchCalculator
            self._batch = BatchCalculator(param_path=self.parameters["param_path"], device=self.parameters["device"],
                                          learned_guess=self.parameters["learned_guess"],
                                          spin_multiplicity=self.parameters["multiplicity"],
                                          level_shift=self.parameters["level_shift"], **self._options())
        return self._batch

    @staticmethod
    def _numbers_positions(atoms):
        if atoms is None:
            raise RuntimeError("no ASE Atoms object supplied or attached")
        if any(np.asarray(atoms.get_pbc()).tolist()):
            raise ValueError("the B200 engine supports non-periodic systems only")
        return (np.asarray(atoms.get_atomic_numbers(), dtype=np.int64),
                np.asarray(atoms.get_positions(), dtype=float).reshape(-1, 3))

    def calculate(self, atoms=None, properties=("energy",), system_changes=all_changes) -> None:
        """Single point into ``self.results`` in ASE units (reference ``ase.py:358-434``)."""
        _AseCalculator.calculate(self, atoms, properties, system_changes)
        numbers, positions = self._numbers_positions(self.atoms)
        need_forces = "forces" in set(properties)
        res = self._batch_calc().calculate([(numbers, positions)], unit="angstrom",
                                           charges=np.array([float(self.parameters["charge"])]),
                                           compute_gradient=need_forces, raise_on_error=True)
        self.results.update(self._results_of(res, 0, need_forces))

    def calculate_many(self, structures, properties=("energy", "forces")) -> list[dict]:
        """Evaluates many structures in one batched engine call; returns one
        results dict (ASE units plus native_* keys) per structure."""
        mols = [self._numbers_positions(a) for a in structures]
        need_forces = "forces" in set(properties)
        charges = np.full(len(mols), float(self.parameters["charge"]))
        res = self._batch_calc().calculate(mols, unit="angstrom", charges=charges, compute_gradient=need_forces,
                                           raise_on_error=True)
        return [self._results_of(res, m, need_forces) for m in range(len(mols))]

    @staticmethod
    def _results_of(res, m, need_forces) -> dict:
        from ._lib import TERM_NAMES
        a0, a1 = int(res.atom_offsets[m]), int(res.atom_offsets[m + 1])
        terms = {k: float(v) for k, v in zip(TERM_NAMES, res.terms[m])}
        dip = np.asarray(res.dipole[m], dtype=float)
        out = {
            "energy": float(res.energy[m]) * _ENERGY,
            "charges": np.asarray(res.atomic_charges[a0:a1], dtype=float),
            "dipole": dip * _DIPOLE,
            "native_dipole_au": dip,
            "native_energy_terms_hartree": terms,
            "native_energy_terms_ev": {k: v * _ENERGY for k, v in terms.items()},
            "native_converged": bool(res.status[m] == 0),
            "native_iterations": int(res.iterations[m]),
        }
        if need_forces and res.gradient is not None:
            f = -np.asarray(res.gradient[a0:a1], dtype=float)
            out["native_forces_hartree_per_bohr"] = f
            out["forces"] = f * _FORCE
        return out

    def native_calculator(self) -> Gfn1NativeCalculator:
        """The atomic-unit single-molecule calculator with the same options."""
        if self._native is None:
            opts = self._options()
            self._native = Gfn1NativeCalculator(param_path=self.parameters["param_path"],
                                                charge=self.parameters["charge"], device=self.parameters["device"],
                                                multiplicity=self.parameters["multiplicity"],
                                                level_shift=self.parameters["level_shift"], **opts)
        return self._native

    def get_dipole_au(self, atoms=None):
        """Mulliken dipole in e*bohr (reference ``ase.py:571-580``)."""
        atoms = self.atoms if atoms is None else atoms
        numbers, positions = self._numbers_positions(atoms)
        return np.asarray(self.native_calculator().calculate(numbers.tolist(), positions.tolist()).dipole)

    def get_hessian(self, atoms=None):
        """Nuclear Hessian d2E/dR_a dR_b as a (3N, 3N) array in eV/Angstrom^2,
        atom-major (reference ``ase.py:641-672``, non-periodic).  Central
        differences of the engine's analytic gradient, all 6N displacements in
        one batched engine call (``gfn1_rs.hessian``)."""
        from .hessian import hessian_batch
        from .native import ANGSTROM_TO_BOHR

        atoms = self.atoms if atoms is None else atoms
        numbers, positions = self._numbers_positions(atoms)
        out = hessian_batch(self._batch_calc(), [0, len(numbers)], numbers, positions * ANGSTROM_TO_BOHR,
                            charges=[float(self.parameters["charge"])])
        if out["hessians"][0] is None:
            raise RuntimeError(f"Hessian evaluation failed (status {int(out['status'][0])})")
        return out["hessians"][0] * (_HARTREE / _BOHR ** 2)

    def get_vibrational_frequencies(self, atoms=None):
        """Harmonic analysis (reference ``ase.py:674-690``): ``wavenumbers`` in
        cm^-1 (imaginary as negative), ``energies_ev`` (the same quanta in eV)
        and ``modes`` (Cartesian normal-mode displacements, one per row)."""
        from .hessian import hessian_batch, vibrational_analysis
        from .native import ANGSTROM_TO_BOHR

        atoms = self.atoms if atoms is None else atoms
        numbers, positions = self._numbers_positions(atoms)
        out = hessian_batch(self._batch_calc(), [0, len(numbers)], numbers, positions * ANGSTROM_TO_BOHR,
                            charges=[float(self.parameters["charge"])])
        if out["hessians"][0] is None:
            raise RuntimeError(f"Hessian evaluation failed (status {int(out['status'][0])})")
        vib = vibrational_analysis(out["hessians"][0], numbers)
        vib["energies_ev"] = vib["wavenumbers"] * _INVCM_EV
        return vib


__all__ = ["GFN1RSCalculator", "HAVE_ASE"]
