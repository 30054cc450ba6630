"""TBTK's JSON serialization of the KPM path's results.

The C ABI and ``kpm.py`` return plain arrays.  This module writes them in the
text that TBTK's own ``serialize(Serializable::Mode::JSON)`` produces for
the same property, so a program built on TBTK can read the results with
its deserializing constructors, e.g. ``Property::LDOS(text, Mode::JSON)``,
and tools that read TBTK's JSON files read these too.  It also reads such
text back into arrays.

Formats followed (reference files):

* ``Property::LDOS`` -- ``{"energyResolvedProperty": ..., "id": "LDOS"}``
  (Lib/src/Property/LDOS.cpp:121-140);
* ``Property::GreensFunction`` -- it has no serializer of its own, so the
  text is its ``EnergyResolvedProperty`` base and the Green's function type
  is not stored (Lib/include/TBTK/Property/EnergyResolvedProperty.h:1156-1212);
* ``Property::Density`` -- ``{"abstractProperty": ..., "id": "Density"}``
  (Lib/src/Property/Density.cpp:111-130);
* ``AbstractProperty`` -- index descriptor, block size, every datum as the
  string ``std::ostream << value`` gives (six significant digits; complex
  values as ``(re,im)``) (Lib/include/TBTK/Property/AbstractProperty.h:922-954,
  Lib/include/Utilities/TBTK/Serializable.h:464-520);
* ``IndexDescriptor`` of format Custom with its ``IndexTree``
  (Lib/src/Property/IndexDescriptor.cpp:482-539, Lib/src/Core/IndexTree.cpp:
  166-330,606-652) and the energy ``Range`` (Lib/src/Utilities/Range.cpp:
  30-57,94-113);
* the JSON text itself as nlohmann::json 2.1.1 dumps it (json/TBTK/json.hpp:
  keys in byte order, no spaces, doubles as ``%.15g`` with ``.0`` appended
  to integer-like values, non-finite doubles as ``null``).

TBTK has no JSON form for ``SpinPolarizedLDOS`` and ``Magnetization``: their
data are ``SpinMatrix`` values, whose serializer is
``TBTKNotYetImplemented`` (Serializable.h:252-254).  They are not written
here either.

The reference leaves ``defaultValue`` of real-valued properties
uninitialised (the constructors from an IndexTree do not set it), so its
text carries whatever the memory held; this module writes ``"0"``.
"""
import json
import math

import numpy as np

__all__ = ["IndexTree", "dumps", "ldos_json", "ldos_json_patterns", "expand_patterns",
           "greens_function_json", "density_json", "loads", "IDX_ALL", "IDX_SUM_ALL"]

# TBTK's wildcard subindices (Lib/include/Core/TBTK/Subindex.h:395-399), as
# the 32-bit ints they are stored as.
def _i32(v):
    return v - (1 << 32) if v & 0x80000000 else v


IDX_ALL = _i32(0xBFFFFFFF & ~0x20000000)
IDX_SUM_ALL = _i32(0xBFFFFFFF & ~0x20000001)
IDX_SPIN = _i32(0xBFFFFFFF & ~0x20000002)


# --------------------------------------------------------------- JSON text

def _float_text(x):
    """A double as nlohmann::json 2.1.1's serializer writes it."""
    x = float(x)
    if not math.isfinite(x):
        return "null"
    if x == 0:
        return "-0.0" if math.copysign(1.0, x) < 0 else "0.0"
    s = "%.15g" % x
    if "." not in s and "e" not in s:
        s += ".0"
    return s


def dumps(obj):
    """Compact JSON text with nlohmann::json 2.1.1's layout: object keys in
    byte order, no whitespace, its double format."""
    if isinstance(obj, dict):
        keys = sorted(obj, key=lambda k: k.encode())
        return "{" + ",".join(json.dumps(k) + ":" + dumps(obj[k]) for k in keys) + "}"
    if isinstance(obj, (list, tuple)):
        return "[" + ",".join(dumps(v) for v in obj) + "]"
    if isinstance(obj, (bool, np.bool_)):
        return "true" if obj else "false"
    if isinstance(obj, (int, np.integer)):
        return str(int(obj))
    if isinstance(obj, (float, np.floating)):
        return _float_text(obj)
    if isinstance(obj, str):
        return json.dumps(obj)
    raise TypeError(f"cannot serialize {type(obj).__name__}")


def _datum_real(x):
    """``std::stringstream << double`` at the default precision 6."""
    return "%g" % float(x)


def _datum_complex(z):
    """``std::stringstream << std::complex<double>``: ``(re,im)``."""
    z = complex(z)
    return "(%g,%g)" % (z.real, z.imag)


def _parse_real(s):
    return float(s)


def _parse_complex(s):
    s = s.strip()
    if not (s.startswith("(") and s.endswith(")")):
        return complex(float(s), 0.0)
    re, im = s[1:-1].split(",")
    return complex(float(re), float(im))


# --------------------------------------------------------------- IndexTree

def _flatten(index):
    """A TBTK Index as a flat list of subindices; a compound index, given as
    a tuple of tuples ``((to...), (from...))``, gets an IDX_SEPARATOR
    (marked None here) between its parts, as ``Index({to, from})`` does."""
    if len(index) and all(isinstance(p, (tuple, list)) for p in index):
        flat = []
        for n, part in enumerate(index):
            if n:
                flat.append(None)
            flat.extend(int(v) for v in part)
        return flat
    return [int(v) for v in index]


class IndexTree:
    """TBTK's ``IndexTree`` (Lib/src/Core/IndexTree.cpp): non-negative
    subindices, compound indices with separators and, with
    ``wildcards=True``, wildcard subindices (a node whose subindex is a
    wildcard keeps one child, 0, and the wildcard's value as its type).
    Without it negative subindices are rejected."""

    def __init__(self):
        self.children = []
        self.index_included = False
        self.wildcard_index = False
        self.wildcard_type = 0
        self.index_separator = False
        self.linear_index = -1
        self.size = -1

    def add(self, index, wildcards=False):
        """IndexTree::add (IndexTree.cpp:166-306), with its error checks
        raised as ValueError."""
        flat = _flatten(index)
        if not wildcards:
            for v in flat:
                if v is not None and v < 0:
                    raise ValueError(f"index {tuple(index)}: wildcard subindices are not "
                                     f"supported")
        self._add(flat, 0, index)

    def _add(self, flat, sub, index):
        if sub < len(flat):
            v = flat[sub]
            if v is None:
                if self.children and not self.index_separator:
                    raise ValueError(f"index {index}: conflicting index separator at "
                                     f"subindex {sub}")
                self.index_separator = False
                self._add(flat, sub + 1, index)
                self.index_separator = True
                return
            if self.index_separator:
                raise ValueError(f"index {index}: conflicting index separator at "
                                 f"subindex {sub}")
            if v < 0:
                if not self.wildcard_index:
                    if self.children:
                        raise ValueError(f"index {index}: wildcard at subindex {sub} where "
                                         f"concrete indices were added")
                    self.wildcard_index = True
                    self.wildcard_type = v
                if v != self.wildcard_type:
                    raise ValueError(f"index {index}: another wildcard type at subindex {sub}")
                v = 0
            elif self.wildcard_index:
                raise ValueError(f"index {index}: a wildcard was added at subindex {sub}")
            while len(self.children) <= v:
                self.children.append(IndexTree())
            if self.index_included:
                raise ValueError(f"index {index} incompatible with an index added before, "
                                 f"at subindex {sub}")
            self.children[v]._add(flat, sub + 1, index)
        else:
            if self.children:
                raise ValueError(f"index {index} incompatible with an index added before, "
                                 f"at subindex {sub}")
            self.index_included = True

    def generate_linear_map(self):
        """IndexTree::generateLinearMap (IndexTree.cpp:308-330): leaves in
        depth-first order, children by ascending subindex."""
        self.size = self._linear(0)

    def _linear(self, i):
        if not self.children:
            if self.index_included:
                self.linear_index = i
                return i + 1
            return i
        for c in self.children:
            i = c._linear(i)
        return i

    def linear_index_of(self, index):
        """IndexTree::getLinearIndex with SearchMode::MatchWildcards: a
        wildcard node matches any subindex."""
        node = self
        for v in _flatten(index):
            if v is None:
                continue
            if node.wildcard_index:
                v = 0
            if v < 0 or v >= len(node.children):
                raise KeyError(index)
            node = node.children[v]
        if not node.index_included:
            raise KeyError(index)
        return node.linear_index

    def indices(self):
        """The included indices in linear order (flat subindex tuples; a
        separator shows as None)."""
        out = []

        def walk(node, prefix):
            if not node.children:
                if node.index_included:
                    out.append(tuple(prefix))
                return
            for n, c in enumerate(node.children):
                v = node.wildcard_type if node.wildcard_index else n
                walk(c, prefix + ([None] if node.index_separator else []) + [v])

        walk(self, [])
        return out

    def to_json(self):
        """IndexTree::serialize in Mode::JSON (IndexTree.cpp:627-644)."""
        j = {}
        if self.children:
            j["children"] = [c.to_json() for c in self.children]
        j.update({"id": "IndexTree", "indexIncluded": self.index_included,
                  "wildcardIndex": self.wildcard_index, "wildcardType": self.wildcard_type,
                  "indexSeparator": self.index_separator, "linearIndex": self.linear_index,
                  "size": self.size})
        return j

    @classmethod
    def from_json(cls, j):
        t = cls()
        t.children = [cls.from_json(c) for c in j.get("children", [])]
        t.index_included = bool(j["indexIncluded"])
        t.wildcard_index = bool(j["wildcardIndex"])
        t.wildcard_type = int(j["wildcardType"])
        t.index_separator = bool(j["indexSeparator"])
        t.linear_index = int(j["linearIndex"])
        t.size = int(j["size"])
        return t


def _tree(indices):
    if len(indices) == 0:
        raise ValueError("no indices")
    tree = IndexTree()
    for idx in indices:
        tree.add(idx)
    tree.generate_linear_map()
    if tree.size != len(indices):
        raise ValueError("an index is given more than once")
    return tree


# --------------------------------------------------------------- properties

def _window(lower, upper, resolution):
    """The PropertyExtractor's inclusive ``Range(lower, upper, resolution)``
    (Range.cpp:30-57) as Range::serialize writes it."""
    resolution = int(resolution)
    if resolution <= 1:
        raise ValueError("'resolution' must be larger than 1.")
    dx = (float(upper) - float(lower)) / (resolution - 1)
    return {"id": "Range", "start": float(lower), "dx": dx, "resolution": resolution}


def _abstract(tree, block, data, datum, default):
    return {"id": "AbstractProperty",
            "indexDescriptor": {"id": "IndexDescriptor", "format": "Custom",
                                "indexTree": tree.to_json()},
            "blockSize": int(block),
            "data": [datum(v) for v in data],
            "allowIndexOutOfBoundsAccess": False,
            "defaultValue": default}


def _blocks(tree, indices, values, dtype):
    """values[k] (one block per index k) placed at the tree's linear order."""
    values = np.asarray(values, dtype=dtype)
    if values.ndim == 1:
        values = values[:, None]
    if values.shape[0] != len(indices):
        raise ValueError(f"{len(indices)} indices but {values.shape[0]} data blocks")
    out = np.zeros((len(indices), values.shape[1]), dtype=dtype)
    for k, idx in enumerate(indices):
        out[tree.linear_index_of(idx)] = values[k]
    return out.reshape(-1)


def _energy_resolved(tree, indices, values, lower, upper, dtype, datum, default):
    values = np.asarray(values, dtype=dtype)
    if values.ndim != 2:
        raise ValueError("energy-resolved data must be [indices][energies]")
    win = _window(lower, upper, values.shape[1])
    data = _blocks(tree, indices, values, dtype)
    return {"id": "EnergyResolvedProperty", "energyType": "Real", "energyWindow": win,
            "abstractProperty": _abstract(tree, values.shape[1], data, datum, default)}


def ldos_json(indices, ldos, lower, upper):
    """``Property::LDOS`` text of ldos[k][e] at indices[k] (index tuples),
    on the PropertyExtractor's inclusive energy window (lower, upper,
    ldos.shape[1] points), as ``calculateLDOS(patterns)`` lays it out
    (PropertyExtractor/ChebyshevExpander.cpp:475-505)."""
    tree = _tree(indices)
    erp = _energy_resolved(tree, indices, ldos, lower, upper, np.float64, _datum_real, "0")
    return dumps({"id": "LDOS", "energyResolvedProperty": erp})


def _matches(pattern, index):
    return len(pattern) == len(index) and all(
        p < 0 or p == v for p, v in zip(pattern, index))


def expand_patterns(patterns, model_indices):
    """The concrete indices of the model that calculateLDOS(patterns)
    computes, in the order it visits them: every model index that matches
    a pattern (IDX_ALL and IDX_SUM_ALL match any value), in index-tree
    order (PropertyExtractor::generateIndexTree,
    Lib/src/PropertyExtractor/PropertyExtractor.cpp:323-420, with the
    summation wildcards expanded).  model_indices: every index of the model
    (its HoppingAmplitudeSet's basis), as tuples."""
    pats = [tuple(int(v) for v in p) for p in patterns]
    for p in pats:
        for v in p:
            if v < 0 and v not in (IDX_ALL, IDX_SUM_ALL):
                raise ValueError(f"pattern {p}: only IDX_ALL and IDX_SUM_ALL wildcards are "
                                 f"read here")
    model = [tuple(int(v) for v in i) for i in model_indices]
    tree = IndexTree()
    for p in pats:
        for idx in model:
            if _matches(p, idx):
                tree.add(idx)
    tree.generate_linear_map()
    return tree.indices()


def ldos_json_patterns(patterns, model_indices, ldos, lower, upper):
    """``Property::LDOS`` text of ``calculateLDOS(patterns)``
    (PropertyExtractor/ChebyshevExpander.cpp:475-505): entries for the
    patterns' matches with IDX_SUM_ALL subindices kept as wildcards
    (generateIndexTree with keepSummationWildcards), and the LDOS of each
    concrete index added into its entry in expand_patterns order, as the
    reference's calculate() loop does (PropertyExtractor.h:856-900).
    ldos: mapping from each index of expand_patterns to its LDOS [E]."""
    pats = [tuple(int(v) for v in p) for p in patterns]
    concrete = expand_patterns(pats, model_indices)
    layout = IndexTree()
    for p in pats:
        for idx in concrete:
            if _matches(p, idx):
                layout.add(tuple(IDX_SUM_ALL if v == IDX_SUM_ALL else idx[m]
                                 for m, v in enumerate(p)), wildcards=True)
    layout.generate_linear_map()
    if not concrete:
        raise ValueError("the patterns match no index of the model")
    E = np.asarray(ldos[concrete[0]]).size
    win = _window(lower, upper, E)
    data = np.zeros((layout.size, E))
    for idx in concrete:
        row = layout.linear_index_of(idx)
        data[row] += np.asarray(ldos[idx], dtype=np.float64)
    erp = {"id": "EnergyResolvedProperty", "energyType": "Real", "energyWindow": win,
           "abstractProperty": _abstract(layout, E, data.reshape(-1), _datum_real, "0")}
    return dumps({"id": "LDOS", "energyResolvedProperty": erp})


def greens_function_json(to, frm, greens, lower, upper):
    """``Property::GreensFunction`` text of greens[k][e] = G(to[k], frm; E_e),
    laid out as ``calculateGreensFunctions(to, from, type)`` does, with the
    compound indices {to[k], from} (PropertyExtractor/ChebyshevExpander.cpp:
    234-295).  The type is not part of TBTK's text."""
    pairs = [(tuple(t), tuple(frm)) for t in to]
    tree = _tree(pairs)
    erp = _energy_resolved(tree, pairs, greens, lower, upper, np.complex128,
                           _datum_complex, "(0,0)")
    return dumps(erp)


def density_json(indices, density):
    """``Property::Density`` text of density[k] at indices[k]
    (calculateDensity(patterns), PropertyExtractor/ChebyshevExpander.cpp:
    297-327)."""
    tree = _tree(indices)
    data = _blocks(tree, indices, density, np.float64)
    return dumps({"id": "Density", "abstractProperty": _abstract(tree, 1, data, _datum_real,
                                                                 "0")})


def loads(text):
    """Reads the text of an LDOS, GreensFunction or Density (as written by
    TBTK or by this module).  Returns a dict: ``kind`` ("LDOS",
    "GreensFunction" or "Density"), ``indices`` (flat subindex tuples in
    data order; None marks a separator), ``energies`` (None for Density)
    and ``data`` ([indices][block], complex for GreensFunction)."""
    j = json.loads(text)
    kind = j.get("id")
    if kind == "LDOS":
        erp = j["energyResolvedProperty"]
    elif kind == "EnergyResolvedProperty":
        erp, kind = j, "GreensFunction"
    elif kind == "Density":
        erp = None
    else:
        raise ValueError(f"not an LDOS, GreensFunction or Density serialization: {kind!r}")
    ap = (erp or j)["abstractProperty"]
    desc = ap["indexDescriptor"]
    if desc["format"] != "Custom":
        raise ValueError(f"index descriptor format {desc['format']!r} is not read here")
    tree = IndexTree.from_json(desc["indexTree"])
    parse = _parse_complex if kind == "GreensFunction" else _parse_real
    block = int(ap["blockSize"])
    data = np.array([parse(s) for s in ap["data"]],
                    dtype=np.complex128 if kind == "GreensFunction" else np.float64)
    energies = None
    if erp is not None:
        if erp["energyType"] != "Real":
            raise ValueError("only real energy windows are read here")
        w = erp["energyWindow"]
        energies = np.array([w["start"] + k * w["dx"] for k in range(int(w["resolution"]))])
    return {"kind": kind, "indices": tree.indices(), "energies": energies,
            "data": data.reshape(-1, block)}
