"""Per-term gradient probe of the oracle on caffeine, after the reference's
tests/gradient_fd_probe.rs:41-120: at the same (atom, axis) probes and step
h = 1e-4 bohr, the analytic repulsion and D3 gradients against central
differences of their own energies (1e-7 Eh/bohr), and the electronic part of
the gradient (total minus the classical terms) against central differences of
the SCC free energy minus those terms, converged tightly (1e-7 Eh/bohr;
measured 4e-9, 1e-11 and 2e-9)."""
from conftest import smoke_molecule

PROBES = ((0, 1), (0, 2), (1, 1), (1, 2), (2, 2), (3, 2), (6, 1), (8, 1))
H = 1.0e-4
TIGHT = dict(energy_tolerance=1e-10, charge_tolerance=1e-8, max_scc=1000)


def _shifted(x, atom, axis, d):
    y = x.copy()
    y[atom, axis] += d
    return y


def test_classical_terms_match_finite_differences(oracle_mod, fixtures):
    z, x = smoke_molecule(fixtures, "caffeine")
    for name in ("repulsion", "dispersion"):
        _, g = oracle_mod.classical_term(name, z, x)
        for atom, axis in PROBES:
            ep, _ = oracle_mod.classical_term(name, z, _shifted(x, atom, axis, H), gradient=False)
            em, _ = oracle_mod.classical_term(name, z, _shifted(x, atom, axis, -H), gradient=False)
            assert abs(g[atom, axis] - (ep - em) / (2 * H)) <= 1e-7, (name, atom, axis)


def test_electronic_gradient_matches_finite_differences(oracle_mod, fixtures):
    z, x = smoke_molecule(fixtures, "caffeine")
    opt = oracle_mod.make_options(**TIGHT)
    r = oracle_mod.run(z, x, options=opt)
    g_cls = sum(oracle_mod.classical_term(n, z, x)[1] for n in oracle_mod.CLASSICAL_TERMS)
    g_el = r.gradient - g_cls

    def e_el(y):
        t = oracle_mod.run(z, y, options=opt, gradient=False, init_shell_charges=r.shell_charges).terms
        return t["total_free"] - t["repulsion"] - t["dispersion"] - t["halogen"]

    for atom, axis in PROBES:
        fd = (e_el(_shifted(x, atom, axis, H)) - e_el(_shifted(x, atom, axis, -H))) / (2 * H)
        assert abs(g_el[atom, axis] - fd) <= 1e-7, (atom, axis, g_el[atom, axis], fd)
