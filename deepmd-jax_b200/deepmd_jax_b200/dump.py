"""Extended-XYZ trajectory dumps with the reference's file names, options and
frame format (deepmd_jax/md_utils.py:40-256, used by md.py:807-938).

``dump_prefix='traj'`` writes ``traj_position.xyz`` (and ``traj_velocity.xyz``
/ ``traj_centroid.xyz`` for ``dump_content='all'`` or a subset of
('position', 'velocity', 'centroid')); under PIMD the position and velocity
files are split per bead (``traj_position_bead{b}.xyz``).  Each frame is::

    N
    Lattice="Lx 0 0 0 Ly 0 0 0 Lz" Properties=species:S:1:pos:R:3 step=K pbc="T T T"
    O  x y z
    ...

with 8 decimals for float32 data (the engine's arithmetic).  The reference
writes through ASE; this writer produces the same text without it.
"""
from __future__ import annotations

import glob
import os

import numpy as np

KINDS = ("position", "velocity", "centroid")

# chemical symbols by atomic number, for models that store chemical_types
SYMBOLS = ("X H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se Br Kr "
           "Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb "
           "Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No Lr").split()


# The dump_content vocabulary (md_utils.py:30-68): each word names the kinds it
# stands for, without and with beads; a kind name stands for itself.
_CONTENT_WORDS = {
    "all": (("position", "velocity"), KINDS),
    "positions": (("position",), ("position", "centroid")),
}
_DEFAULT_CONTENT = tuple(_CONTENT_WORDS)  # the words allowed without a dump_prefix

_MSG_NOT_ITERABLE = ("dump_content must be 'all', 'positions', a dump kind string, "
                     "or an iterable of dump kind strings.")


def _content_items(dump_content):
    """dump_content as a tuple of entries: one string is one entry."""
    if isinstance(dump_content, str):
        return (dump_content,)
    try:
        return tuple(dump_content)
    except TypeError as exc:
        raise ValueError(_MSG_NOT_ITERABLE) from exc


def normalize_content(dump_content, n_bead):
    """The kinds a dump_content asks for, in file order (md_utils.py:30-68):
    words expand through _CONTENT_WORDS for a run with or without beads, kind
    names stand for themselves, and the union is checked against KINDS."""
    pimd = n_bead > 1
    items = _content_items(dump_content)
    if not items:
        raise ValueError("dump_content must not be empty when dump_prefix is set.")
    non_str = [x for x in items if not isinstance(x, str)]
    if non_str:
        raise ValueError("dump_content entries must be strings; got %r." % (non_str,))
    wanted = set()
    for item in items:
        wanted.update(_CONTENT_WORDS[item][pimd] if item in _CONTENT_WORDS else (item,))
    unknown = sorted(wanted.difference(KINDS))
    if unknown:
        raise ValueError("Unknown dump_content entries %s. Allowed entries are %s, 'positions', or 'all'."
                         % (unknown, list(KINDS)))
    if not pimd and "centroid" in wanted:
        raise ValueError("dump_content includes 'centroid', which is only meaningful when n_bead > 1.")
    return tuple(filter(wanted.__contains__, KINDS))


def _bead_path(path, bead):
    root, ext = os.path.splitext(path)
    return "%s_bead%d%s" % (root, bead, ext)


def prepare(type_idx, type_symbols, n_bead, default_interval, dump_interval=None, dump_prefix=None,
            dump_content="positions", dump_mode="overwrite"):
    """[(kind, path, symbols, bead or None)] and the write interval
    (md_utils.py:194-229); ([], None) when nothing is dumped."""
    if dump_prefix is None:
        # without a prefix only the default words are accepted, and nothing is written
        if isinstance(dump_content, str) and dump_content in _DEFAULT_CONTENT:
            return [], None
        raise ValueError("dump_content requires dump_prefix to be set.")
    prefix = os.fspath(dump_prefix)
    if not prefix:
        raise ValueError("dump_prefix must be a non-empty path prefix.")
    kinds = normalize_content(dump_content, n_bead)
    if dump_mode not in ("overwrite", "append"):
        raise ValueError("dump_mode must be 'overwrite' or 'append'; got %r" % (dump_mode,))
    if type_symbols is None:
        raise ValueError("Simulation.run(dump_prefix=...) requires `type_symbols=[...]` at Simulation(...) "
                         "construction so XYZ output can label atoms.")
    interval = int(dump_interval) if dump_interval is not None else int(default_interval)
    if interval <= 0:
        raise ValueError("dump_interval must be positive; got %d" % interval)
    symbols = [str(s) for s in np.array(type_symbols, dtype=object)[np.asarray(type_idx)]]
    dumps = []
    for kind in kinds:
        path = "%s_%s.xyz" % (prefix, kind)
        split = n_bead > 1 and kind != "centroid"
        if dump_mode == "overwrite":
            if os.path.exists(path):
                os.remove(path)
            if split:
                root, ext = os.path.splitext(path)
                for p in glob.glob("%s_bead*%s" % (root, ext)):
                    os.remove(p)
        if split:
            dumps += [(kind, _bead_path(path, b), symbols, b) for b in range(n_bead)]
        else:
            dumps.append((kind, path, symbols, None))
    return dumps, interval


def write_frame(dumps, pos, vel, centroid, box, step=None):
    """Append one frame to every dump file (md_utils.py:119-136, 232-256).
    pos / vel: (N, 3) or (P, N, 3); centroid (N, 3); box (3,)."""
    L = np.asarray(box, dtype=np.float64).reshape(3)
    lattice = " ".join("%.8f" % v for v in np.diag(L).reshape(9))
    src = {"position": pos, "velocity": vel, "centroid": centroid}
    for kind, path, symbols, bead in dumps:
        data = src[kind]
        if data is None:
            raise ValueError("Missing %s frame for XYZ dump." % kind)
        data = np.asarray(data)
        if bead is not None:
            data = data[bead]
        elif data.ndim == 3:
            data = data.reshape(-1, 3)
        head = ['Lattice="%s"' % lattice, "Properties=species:S:1:pos:R:3"]
        if step is not None:
            head.append("step=%d" % int(step))
        head.append('pbc="T T T"')
        lines = ["%d\n" % len(symbols), " ".join(head) + "\n"]
        lines += ["%-2s %.8f %.8f %.8f\n" % (s, x[0], x[1], x[2]) for s, x in zip(symbols, data)]
        with open(path, "a", encoding="utf-8") as fh:
            fh.write("".join(lines))


def read_xyz(path):
    """Frames of a file written by write_frame: list of (symbols, (N, 3),
    comment) - a reader for tests and users without ASE."""
    frames = []
    with open(path, encoding="utf-8") as fh:
        lines = fh.read().splitlines()
    i = 0
    while i < len(lines):
        n = int(lines[i])
        comment = lines[i + 1]
        rows = [ln.split() for ln in lines[i + 2:i + 2 + n]]
        frames.append(([r[0] for r in rows], np.array([[float(v) for v in r[1:4]] for r in rows]), comment))
        i += 2 + n
    return frames
