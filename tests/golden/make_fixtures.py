"""Regenerate the golden fixtures of this directory from the eT source tree.

Run in a container that has the eT sources mounted (read-only is fine):

    python tests/golden/make_fixtures.py /path/to/eT

It writes

* ``basis_cc-pvdz.json``, ``basis_sto-3g.json`` - the cc-pVDZ and STO-3G shells of H, He and O,
  taken from ``ao_basis/*.g94`` (published basis data; STO-3G's SP shells split into an s and a p
  shell), so the oracle's
  integral front end can rebuild eT's test molecules without the eT tree;
* ``et_reference_values.json`` - numbers parsed from eT's committed
  regression outputs (``tests/*/result/*.out``): geometries, HF energies,
  the (E, |Omega|) history of the DIIS ground-state solver, final CCSD
  energies, the number of Cholesky vectors and EOM-CCSD excitation energies;
* ``et_restart_h2o_he.npz`` - the vectors eT itself wrote for H2O+He/cc-pVDZ
  (``tests/restart_ccsd_v1.0/old_restart_files``, eT 1.0 record files, read with
  ``et_b200.restart``): MO coefficients and energies, converged amplitudes t,
  multipliers tbar, and three right/left EOM-CCSD eigenvectors with their
  excitation energies.

Nothing here is executed by the tests; they only read the files written.
"""

from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _geometry(inp: str):
    m = re.search(r"geometry\s*\n\s*basis:\s*(\S+)\s*\n(.*?)end geometry", inp, re.S | re.I)
    atoms = []
    for line in m.group(2).strip().splitlines():
        tok = line.split()
        atoms.append([tok[0], float(tok[1]), float(tok[2]), float(tok[3])])
    return m.group(1).lower(), atoms


def _gs_history(out: str):
    block = out.split("Iteration    Energy (a.u.)        |omega|")[1].split("Convergence criterion")[0]
    hist = []
    for line in block.splitlines():
        tok = line.split()
        if len(tok) == 4 and tok[0].isdigit():
            hist.append([float(tok[1]), float(tok[2])])
    return hist


def _scf_energy(out: str):
    return float(re.search(r"Total energy:\s+(-?\d+\.\d+)", out).group(1))


def _final_cc(out: str):
    return float(re.search(r"Final ground state energy \(a\.u\.\):\s+(-?\d+\.\d+)", out).group(1))


def _n_cholesky(out: str):
    return int(re.search(r"Final number of Cholesky vectors:\s+(\d+)", out).group(1))


def _cd_threshold(inp: str):
    m = re.search(r"solver cholesky\s*\n\s*threshold:\s*(\S+)", inp, re.I)
    return float(m.group(1).replace("d", "e").replace("D", "e"))


def _excitations(out: str):
    block = out.split("CCSD excitation energies:")[1].split("eV/Hartree")[0]
    vals = []
    for line in block.splitlines():
        tok = line.split()
        if len(tok) == 3 and tok[0].isdigit():
            vals.append(float(tok[1]))
    return vals


def _test(root, name):
    d = os.path.join(root, "tests", name)
    inp = open(os.path.join(d, name + ".inp")).read()
    out = open(os.path.join(d, "result", name + ".out")).read()
    return inp, out


def _dipole(out: str):
    """The CC dipole table of a mean-value run: electronic / nuclear / total per component, Debye."""
    block = out[out.index("Dipole moment in [Debye]"):]
    conv = float(re.search(r"Conversion factor from Debye a\.u\.:\s+(\S+)", block).group(1))
    rows = {}
    for comp in ("x", "y", "z"):
        m = re.search(r"\n\s+%s\s+(-?\d+\.\d+)\s+(-?\d+\.\d+)\s+(-?\d+\.\d+)" % comp, block)
        rows[comp] = [float(m.group(k)) for k in (1, 2, 3)]
    return dict(debye_per_au=1.0 / conv, au_per_debye=conv, electronic=[rows[c][0] for c in "xyz"],
                nuclear=[rows[c][1] for c in "xyz"], total=[rows[c][2] for c in "xyz"])


def _restart_vectors(d: str) -> None:
    import numpy as np
    from et_b200 import restart as rs
    n_o, n_v, n_gs, n_es = rs.read_legacy_cc_dimensions(os.path.join(d, "cc_restart_file"))
    n_ao = int.from_bytes(rs.read_records(os.path.join(d, "scf_restart_file"))[0], "little")
    C, eps = rs.read_legacy_orbitals(d, n_ao)
    w = rs.read_legacy_excitation_energies(os.path.join(d, "excitation_energies"))
    vec = lambda name: rs.read_legacy_vector(os.path.join(d, name))
    np.savez(os.path.join(HERE, "et_restart_h2o_he.npz"),
             source=np.array("tests/restart_ccsd_v1.0/old_restart_files"),
             n_o=n_o, n_v=n_v, C=C, eps=eps, t=vec("t"), tbar=vec("tbar"), omega=w,
             r=np.stack([vec(f"r_{k + 1:03d}") for k in range(w.size)]),
             l=np.stack([vec(f"l_{k + 1:03d}") for k in range(w.size)]))


def main(root: str) -> None:
    values = {}
    for name in ("ccsd_gs_energy", "ccsd_lr_polarizability"):
        inp, out = _test(root, name)
        basis, atoms = _geometry(inp)
        values[name] = dict(
            source=f"tests/{name}/result/{name}.out",
            basis=basis, atoms=atoms, cd_threshold=_cd_threshold(inp),
            e_hf=_scf_energy(out), e_ccsd=_final_cc(out), n_cholesky=_n_cholesky(out),
            gs_history=_gs_history(out),
        )
    for name in ("ccsd_right_es_energies", "ccsd_left_es_energies"):
        inp, out = _test(root, name)
        basis, atoms = _geometry(inp)
        values[name] = dict(source=f"tests/{name}/result/{name}.out", basis=basis, atoms=atoms,
                            cd_threshold=_cd_threshold(inp), e_ccsd=_final_cc(out),
                            excitation_energies=_excitations(out))
    name = "restart_ccsd_v1.0"
    inp, out = _test(root, name)
    basis, atoms = _geometry(inp)
    values[name] = dict(source=f"tests/{name}/result/{name}.out", basis=basis, atoms=atoms,
                        cd_threshold=_cd_threshold(inp), e_ccsd=_final_cc(out),
                        excitation_energies=_excitations(out))
    name = "ccsd_dipole"
    inp, out = _test(root, name)
    basis, atoms = _geometry(inp)
    values[name] = dict(source=f"tests/{name}/result/{name}.out", basis=basis, atoms=atoms,
                        cd_threshold=_cd_threshold(inp), e_hf=_scf_energy(out), e_ccsd=_final_cc(out),
                        n_cholesky=_n_cholesky(out), dipole_debye=_dipole(out))
    with open(os.path.join(HERE, "et_reference_values.json"), "w") as f:
        json.dump(values, f, indent=1)

    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    _restart_vectors(os.path.join(root, "tests", "restart_ccsd_v1.0", "old_restart_files"))
    from oracle.frontend import parse_g94
    for bname in ("cc-pvdz", "sto-3g"):
        text = open(os.path.join(root, "ao_basis", bname + ".g94")).read()
        basis = parse_g94(text, {"H", "He", "O"})
        with open(os.path.join(HERE, f"basis_{bname}.json"), "w") as f:
            json.dump({"source": f"ao_basis/{bname}.g94", "shells": basis}, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <path to the eT source tree>")
    main(sys.argv[1])
