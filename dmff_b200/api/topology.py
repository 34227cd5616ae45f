"""Topology for the drop-in API: atoms, residues, bonds, periodic box, covalent map.

Mirrors the parts of dmff/api/topology.py that the ADMP / classical generators read
(``atoms()``, ``getNumAtoms()``, ``getPeriodicBoxVectors()``, ``bonds()``, atom ``meta``
type/class labels, ``buildCovMat`` at topology.py:391-418).  OpenMM is not a dependency:
``PDBFile`` reads ATOM/HETATM/CRYST1 records, and residue templates from force-field XML
assign atom types and template bonds by atom name.

``buildCovMat`` returns a sparse ``CovalentMap``: the reference's dense N x N integer matrix
(1..nmax = bond-path length, 0 = not bonded) costs O(N^2) memory (80 GB at 100k atoms); the
sparse form answers ``cov_map[i, j]`` with the same values and exports (i, j, nbond) rows.
"""
from collections import deque

import numpy as np


class Atom:
    def __init__(self, index, name, element, residue):
        self.index = index
        self.name = name
        self.element = element
        self.residue = residue
        self.meta = {}


class Residue:
    def __init__(self, index, name):
        self.index = index
        self.name = name
        self._atoms = []

    def atoms(self):
        return iter(self._atoms)


class Bond:
    def __init__(self, atom1, atom2):
        self.atom1 = atom1
        self.atom2 = atom2


class CovalentMap:
    """Sparse topological-distance map: ``cm[i, j]`` -> shortest bond path length (<= nmax) or 0."""

    def __init__(self, n_atoms, rows):
        self.n_atoms = n_atoms
        rows = np.asarray(rows, dtype=np.int64).reshape(-1, 3)
        # keep both orientations, sorted by (i, j) for searchsorted lookups
        both = np.concatenate([rows, rows[:, [1, 0, 2]]], axis=0) if len(rows) else rows
        order = np.lexsort((both[:, 1], both[:, 0])) if len(both) else np.zeros(0, dtype=np.int64)
        self._rows = both[order]
        self._keys = self._rows[:, 0] * n_atoms + self._rows[:, 1] if len(both) else np.zeros(0, np.int64)
        self.shape = (n_atoms, n_atoms)

    def pairs(self):
        """(i, j, nbond) rows with i < j."""
        r = self._rows
        return r[r[:, 0] < r[:, 1]].copy()

    def neighbors(self, i, d=1):
        lo = np.searchsorted(self._keys, i * self.n_atoms)
        hi = np.searchsorted(self._keys, (i + 1) * self.n_atoms)
        r = self._rows[lo:hi]
        return r[r[:, 2] == d, 1]

    def lookup(self, i, j):
        i = np.asarray(i, dtype=np.int64)
        j = np.asarray(j, dtype=np.int64)
        out = np.zeros(np.broadcast(i, j).shape, dtype=np.int64)
        valid = (i >= 0) & (j >= 0) & (i < self.n_atoms) & (j < self.n_atoms)
        if len(self._keys) == 0:
            return out
        key = np.where(valid, i * self.n_atoms + j, -1)
        pos = np.searchsorted(self._keys, key)
        pos = np.clip(pos, 0, len(self._keys) - 1)
        hit = valid & (self._keys[pos] == key)
        out[hit] = self._rows[pos[hit], 2]
        return out

    def __getitem__(self, idx):
        i, j = idx
        return self.lookup(i, j)

    def dense(self):
        m = np.zeros((self.n_atoms, self.n_atoms), dtype=np.int64)
        if len(self._rows):
            m[self._rows[:, 0], self._rows[:, 1]] = self._rows[:, 2]
        return m


def covalent_rows(n_atoms, bonds, nmax=6):
    """Shortest bond-path lengths 1..nmax between atoms (topology.py:391-411 semantics), by BFS."""
    adj = [[] for _ in range(n_atoms)]
    for a, b in bonds:
        adj[a].append(b)
        adj[b].append(a)
    rows = []
    for i in range(n_atoms):
        if not adj[i]:
            continue
        dist = {i: 0}
        q = deque([i])
        while q:
            u = q.popleft()
            if dist[u] >= nmax:
                continue
            for v in adj[u]:
                if v not in dist:
                    dist[v] = dist[u] + 1
                    q.append(v)
        for j, d in dist.items():
            if j > i:
                rows.append((i, j, d))
    return np.asarray(rows, dtype=np.int64).reshape(-1, 3)


class DMFFTopology:
    def __init__(self):
        self._atoms = []
        self._residues = []
        self._bonds = []
        self._box = None  # nm, rows = lattice vectors
        self._meta = {}

    # construction -------------------------------------------------------------------
    def addResidue(self, name):
        r = Residue(len(self._residues), name)
        self._residues.append(r)
        return r

    def addAtom(self, name, element, residue, meta=None):
        a = Atom(len(self._atoms), name, element, residue)
        if meta:
            a.meta.update(meta)
        residue._atoms.append(a)
        self._atoms.append(a)
        return a

    def addBond(self, a1, a2):
        i1 = a1.index if isinstance(a1, Atom) else int(a1)
        i2 = a2.index if isinstance(a2, Atom) else int(a2)
        self._bonds.append(Bond(self._atoms[i1], self._atoms[i2]))

    def setPeriodicBoxVectors(self, box_nm):
        self._box = None if box_nm is None else np.asarray(box_nm, dtype=np.float64).reshape(3, 3)

    # queries (reference names) --------------------------------------------------------
    def atoms(self):
        return iter(self._atoms)

    def residues(self):
        return iter(self._residues)

    def bonds(self):
        return iter(self._bonds)

    def getNumAtoms(self):
        return len(self._atoms)

    def getPeriodicBoxVectors(self):
        return None if self._box is None else self._box.copy()

    def bond_array(self):
        return np.asarray([(b.atom1.index, b.atom2.index) for b in self._bonds], dtype=np.int64).reshape(-1, 2)

    def buildCovMat(self, nmax=6):
        return CovalentMap(self.getNumAtoms(), covalent_rows(self.getNumAtoms(), self.bond_array(), nmax))

    # force-field templates -------------------------------------------------------------
    def apply_templates(self, ffinfo):
        """Assign ``type``/``class`` to atoms from residue templates matched by residue and atom
        names, and add template bonds for residues that have none (a name-based subset of the
        reference's graph-matching TemplateATypeOperator, operators/templatetype.py)."""
        type2class = {t["name"]: t.get("class") for t in ffinfo["AtomTypes"] if "name" in t}
        templates = {r["name"]: r for r in ffinfo["Residues"]}
        have_bond = np.zeros(self.getNumAtoms(), dtype=bool)
        for b in self._bonds:
            have_bond[b.atom1.index] = have_bond[b.atom2.index] = True
        for res in self._residues:
            tpl = templates.get(res.name)
            if tpl is None:
                continue
            by_name = {a.name: a for a in res._atoms}
            names = [p["name"] for p in tpl["particles"]]
            for p in tpl["particles"]:
                a = by_name.get(p["name"])
                if a is None:
                    continue
                # type plus per-atom attributes such as charge; what the caller already set on
                # the atom (as the reference's tests set charges and types by hand) stays
                for k, v in p.items():
                    if k != "name":
                        a.meta.setdefault(k, v)
                a.meta.setdefault("class", type2class.get(a.meta.get("type", p["type"])))
            if not any(have_bond[a.index] for a in res._atoms):
                for b in tpl["bonds"]:
                    if "atomName1" in b:
                        n1, n2 = b["atomName1"], b["atomName2"]
                    elif "from" in b and b["from"].lstrip("-").isdigit():
                        n1, n2 = names[int(b["from"])], names[int(b["to"])]
                    else:
                        n1, n2 = b["from"], b["to"]
                    if n1 in by_name and n2 in by_name:
                        self.addBond(by_name[n1], by_name[n2])
        return self


# water residue / atom name variants that OpenMM's PDB reader maps to the HOH template
_WATER_RES = {"HOH", "WAT", "SOL", "H2O", "TIP3", "TIP", "T3P", "TP3", "SPC"}
_WATER_ATOM = {"OW": "O", "OH2": "O", "HW1": "H1", "HW2": "H2"}


class PDBFile:
    """Minimal PDB reader: ATOM/HETATM records (name, residue, element), CRYST1 box and CONECT
    bonds (deduplicated).  Water residues named SOL/WAT/H2O/TIP3... become HOH with atoms O, H1, H2,
    as OpenMM's reader renames them.  ``positions`` are in nm (numpy [N,3]); ``topology`` is a
    DMFFTopology."""

    def __init__(self, path):
        top = DMFFTopology()
        pos = []
        box = None
        last_key = None
        res = None
        serial = {}
        conect = []
        for line in open(path):
            if line.startswith("CRYST1"):
                a, b, c = float(line[6:15]), float(line[15:24]), float(line[24:33])
                box = np.diag([a, b, c]) / 10.0
            elif line.startswith(("ATOM", "HETATM")):
                name = line[12:16].strip()
                resname = line[17:20].strip()
                if resname in _WATER_RES:
                    resname = "HOH"
                    name = _WATER_ATOM.get(name, name)
                key = (line[21], line[22:27])
                if key != last_key:
                    res = top.addResidue(resname)
                    last_key = key
                elem = line[76:78].strip() or name[0]
                atom = top.addAtom(name, elem, res)
                try:
                    serial[int(line[6:11])] = atom.index
                except ValueError:
                    pass
                pos.append([float(line[30:38]), float(line[38:46]), float(line[46:54])])
            elif line.startswith("CONECT"):
                fields = [line[k:k + 5] for k in range(6, len(line.rstrip()), 5)]
                ids = [int(f) for f in fields if f.strip().isdigit()]
                conect += [(ids[0], o) for o in ids[1:]]
        seen = set()
        for a, b in conect:
            if a in serial and b in serial and a != b:
                i, j = serial[a], serial[b]
                if (min(i, j), max(i, j)) not in seen:
                    seen.add((min(i, j), max(i, j)))
                    top.addBond(i, j)
        top.setPeriodicBoxVectors(box)
        self.topology = top
        self.positions = np.asarray(pos, dtype=np.float64) / 10.0

    def getPositions(self):
        return self.positions
