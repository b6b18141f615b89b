"""eT amplitude files: read and write them so eT and this library can resume from each other.

Current layout (eT 1.x, ``amplitude_file_storer_class.F90:84-160``, a Fortran stream file written
in the machine's byte order, little-endian on x86-64 and aarch64):

    energy (f8) | n_1 (i8) | n_1 values (f8) | n_2 (i8) | n_2 values (f8) ...

one (n, values) pair per block.  CCSD ground-state amplitudes ``t`` and multipliers ``tbar`` have
the blocks [n_t1, n_t2]; excited-state vectors ``r_001``, ``l_001``, ... carry the excitation
energy in the energy field (``file_handling_ccs.F90:147-195``).  Reading stops quietly at the end
of the file after a complete block (eT uses that to start CCSD from CCS singles) and fails on a
block whose length differs from the expected one, as ``read_amplitude_file_storer`` does.

Legacy layout (eT 1.0, described by ``dev_tools/convert_v1_0_restart_files.py:82-183``): Fortran
sequential unformatted records, each framed by a 4-byte length before and after the data.  ``t``
and ``tbar`` hold one record per block, ``r_###``/``l_###`` one record with the whole vector,
``cc_restart_file`` four i8 records (n_o, n_v, n_gs, n_es), ``excitation_energies`` a record with
the number of states and one with the energies, ``orbital_coefficients`` and ``orbital_energies``
one record each (per spin for unrestricted references).
"""

from __future__ import annotations

import os
from typing import Sequence

import numpy as np

_F8 = np.dtype("<f8")
_I8 = np.dtype("<i8")


class RestartFileError(ValueError):
    """A restart file does not have the layout or the sizes expected."""


def ccsd_blocks(n_o: int, n_v: int) -> list[int]:
    """Block sizes of CCSD ground-state and excited-state vectors: [n_t1, n_t2]."""
    n1 = n_o * n_v
    return [n1, n1 * (n1 + 1) // 2]


def save_amplitudes(path: str, vector: np.ndarray, blocks: Sequence[int], energy: float = 0.0) -> None:
    """Write ``vector`` (sum(blocks) values) with its energy in eT's current layout."""
    v = np.ascontiguousarray(vector, dtype=np.float64).ravel()
    if v.size != sum(blocks):
        raise RestartFileError(f"vector has {v.size} values, blocks need {sum(blocks)}")
    with open(path, "wb") as f:
        f.write(np.array([energy], dtype=_F8).tobytes())
        off = 0
        for n in blocks:
            f.write(np.array([n], dtype=_I8).tobytes())
            f.write(v[off:off + n].astype(_F8).tobytes())
            off += n


def read_amplitudes(path: str, blocks: Sequence[int]) -> tuple[np.ndarray, float, int]:
    """Read a file in eT's current layout: (vector, energy, number of values read).

    Values of blocks missing from the end of the file are returned as zero."""
    data = open(path, "rb").read()
    if len(data) < 8:
        raise RestartFileError(f"{path}: too short for the energy field")
    energy = float(np.frombuffer(data[:8], dtype=_F8)[0])
    out = np.zeros(sum(blocks))
    pos, off = 8, 0
    for n in blocks:
        if pos == len(data):
            break                                     # end of file: the remaining blocks are absent
        if pos + 8 > len(data):
            raise RestartFileError(f"{path}: truncated block header at byte {pos}")
        n_file = int(np.frombuffer(data[pos:pos + 8], dtype=_I8)[0])
        if n_file != n:
            raise RestartFileError(f"{path}: wrong number of amplitudes in a block, expected {n}, found {n_file}")
        pos += 8
        if pos + 8 * n > len(data):
            raise RestartFileError(f"{path}: block of {n} values is truncated")
        out[off:off + n] = np.frombuffer(data[pos:pos + 8 * n], dtype=_F8)
        pos += 8 * n
        off += n
    return out, energy, off


def read_records(path: str) -> list[bytes]:
    """Fortran sequential unformatted records (4-byte markers) of an eT 1.0 file."""
    data = open(path, "rb").read()
    recs, pos = [], 0
    while pos < len(data):
        if pos + 4 > len(data):
            raise RestartFileError(f"{path}: truncated record marker at byte {pos}")
        n = int.from_bytes(data[pos:pos + 4], "little")
        end = pos + 4 + n
        if end + 4 > len(data) or int.from_bytes(data[end:end + 4], "little") != n:
            raise RestartFileError(f"{path}: record at byte {pos} is not framed by matching markers")
        recs.append(data[pos + 4:end])
        pos = end + 4
    return recs


def write_records(path: str, records: Sequence[bytes]) -> None:
    """The inverse of :func:`read_records` (used to build eT 1.0 files for tests)."""
    with open(path, "wb") as f:
        for r in records:
            f.write(len(r).to_bytes(4, "little"))
            f.write(r)
            f.write(len(r).to_bytes(4, "little"))


def read_legacy_vector(path: str) -> np.ndarray:
    """All records of an eT 1.0 amplitude file (t, tbar, r_###, l_###) as one vector."""
    return np.concatenate([np.frombuffer(r, dtype=_F8) for r in read_records(path)])


def read_legacy_cc_dimensions(path: str) -> tuple[int, int, int, int]:
    """(n_o, n_v, n_gs_amplitudes, n_es_amplitudes) from an eT 1.0 ``cc_restart_file``."""
    recs = read_records(path)
    if len(recs) < 4:
        raise RestartFileError(f"{path}: expected four records")
    return tuple(int(np.frombuffer(r, dtype=_I8)[0]) for r in recs[:4])


def read_legacy_excitation_energies(path: str) -> np.ndarray:
    recs = read_records(path)
    n = int(np.frombuffer(recs[0], dtype=_I8)[0])
    w = np.frombuffer(recs[1], dtype=_F8)
    if w.size != n:
        raise RestartFileError(f"{path}: {n} states announced, {w.size} energies found")
    return w.copy()


def read_legacy_orbitals(directory: str, n_ao: int) -> tuple[np.ndarray, np.ndarray]:
    """(C (n_ao, n_mo) column-major, orbital energies) of the first spin from an eT 1.0 directory."""
    c = np.frombuffer(read_records(os.path.join(directory, "orbital_coefficients"))[0], dtype=_F8)
    e = np.frombuffer(read_records(os.path.join(directory, "orbital_energies"))[0], dtype=_F8)
    if c.size % n_ao:
        raise RestartFileError(f"orbital coefficients ({c.size} values) do not match n_ao = {n_ao}")
    return c.reshape(n_ao, c.size // n_ao, order="F").copy(), e.copy()


def convert_legacy_directory(old_dir: str, new_dir: str) -> list[str]:
    """Rewrite the CC files of an eT 1.0 restart directory in the current layout.

    Ground-state files get a zero energy and excited-state files their excitation energy, as eT's
    own converter does.  Returns the names written."""
    n_o, n_v, n_gs, n_es = read_legacy_cc_dimensions(os.path.join(old_dir, "cc_restart_file"))
    n1 = n_o * n_v
    n2 = 0 if n_es == n1 else n1 * (n1 + 1) // 2
    gs_blocks = [n1] if n_gs == n1 else [n1, n2]
    es_blocks = [n1] if n2 == 0 else [n1, n2]
    os.makedirs(new_dir, exist_ok=True)
    written = []
    for name in ("t", "tbar"):
        src = os.path.join(old_dir, name)
        if os.path.isfile(src):
            v = read_legacy_vector(src)
            save_amplitudes(os.path.join(new_dir, name), v[:sum(gs_blocks)], gs_blocks, 0.0)
            written.append(name)
    ee_path = os.path.join(old_dir, "excitation_energies")
    if os.path.isfile(ee_path):
        w = read_legacy_excitation_energies(ee_path)
        for k, wk in enumerate(w):
            for side in ("r", "l"):
                name = f"{side}_{k + 1:03d}"
                src = os.path.join(old_dir, name)
                if os.path.isfile(src):
                    save_amplitudes(os.path.join(new_dir, name), read_legacy_vector(src), es_blocks, float(wk))
                    written.append(name)
    return written
