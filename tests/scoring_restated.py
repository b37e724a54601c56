"""Test infrastructure: an independent restatement of smina's pair terms and
of precalculate_linear, to check the engine's host-built tables entry by
entry.  Not used by the product.

Sources restated (reference project paths):
  - term formulas and their parameter syntax: src/lib/everything.h
    (gaussian 48-52, electrostatic 63-104, ad4_solvation 107-154,
    optimal_distance 156-159, gauss 161-187, repulsion 190-217, slope_step
    219-237, hydrophobic / non_hydrophobic 239-299, vdw coefficients
    302-309, vdw 311-363, non_dir_h_bond_lj 367-409, the three quadratic
    h-bond terms 412-510, non_dir_h_bond 513-540, atom_type_* 547-718);
  - type predicates: src/lib/atom_constants.h:240-337 (xs_radius,
    xs_is_hydrophobic / donor / acceptor, xs_h_bond_possible,
    xs_anti_h_bond, string_to_smina_type, solvation_parameter, ad_volume);
  - weighted sum without cutoff test: src/lib/weighted_terms.cpp:51-61;
  - the tables: src/lib/precalculate.h:153-180 (dor and fast from the
    sampled energies) and 195-237 (n = int(factor * cutoff^2) + 3, samples
    at r = sqrt(i / factor)).
The type constants and the builtin functions' terms come from
tests/golden/scoring_ref.json, which tests/golden/make_scoring_ref.py
extracts from the reference's atom_constants.h and builtinscoring.cpp.

Arithmetic follows the reference's operation order in IEEE double; exp is
the C library's (math.exp), as in the C++ code, so the sampled energies can
be compared bit for bit.
"""
import json
import math
import os
import re

import numpy as np

REF = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scoring_ref.json")))
NT = len(REF["types"])
NPAIRS = NT * (NT + 1) // 2
EPS = np.finfo(np.float64).eps

CONF_INDEPENDENT = {"num_tors_add", "num_tors_sqr", "num_tors_sqrt", "num_tors_div", "num_tors_div_simple",
                    "ligand_length", "num_ligands", "num_heavy_atoms_div", "num_heavy_atoms",
                    "num_hydrophobic_atoms", "constant_term"}

# term name -> (parameter regex, charge dependent)
_NUM = r"(\S+)"
PATTERNS = {
    "electrostatic": (rf"electrostatic\(i={_NUM},_\^={_NUM},_c={_NUM}\)", True),
    "ad4_solvation": (rf"ad4_solvation\(d-sigma={_NUM},_s/q={_NUM},_c={_NUM}\)", True),
    "gauss": (rf"gauss\(o={_NUM},_w={_NUM},_c={_NUM}\)", False),
    "repulsion": (rf"repulsion\(o={_NUM},_c={_NUM}\)", False),
    "hydrophobic": (rf"hydrophobic\(g={_NUM},_b={_NUM},_c={_NUM}\)", False),
    "non_hydrophobic": (rf"non_hydrophobic\(g={_NUM},_b={_NUM},_c={_NUM}\)", False),
    "vdw": (rf"vdw\(i={_NUM},_j={_NUM},_s={_NUM},_\^={_NUM},_c={_NUM}\)", False),
    "non_dir_h_bond_lj": (rf"non_dir_h_bond_lj\(o={_NUM},_\^={_NUM},_c={_NUM}\)", False),
    "non_dir_anti_h_bond_quadratic": (rf"non_dir_anti_h_bond_quadratic\(o={_NUM},_c={_NUM}\)", False),
    "donor_donor_quadratic": (rf"donor_donor_quadratic\(o={_NUM},_c={_NUM}\)", False),
    "acceptor_acceptor_quadratic": (rf"acceptor_acceptor_quadratic\(o={_NUM},_c={_NUM}\)", False),
    "non_dir_h_bond": (rf"non_dir_h_bond\(g={_NUM},_b={_NUM},_c={_NUM}\)", False),
    "atom_type_inverse_power": (rf"atom_type_inverse_power\(t1={_NUM},t2={_NUM},i={_NUM},_\^={_NUM},_c={_NUM}\)", False),
    "atom_type_gaussian": (rf"atom_type_gaussian\(t1={_NUM},t2={_NUM},o={_NUM},_w={_NUM},_c={_NUM}\)", False),
    "atom_type_linear": (rf"atom_type_linear\(t1={_NUM},t2={_NUM},g={_NUM},_b={_NUM},_c={_NUM}\)", False),
    "atom_type_quadratic": (rf"atom_type_quadratic\(t1={_NUM},t2={_NUM},o={_NUM},_c={_NUM}\)", False),
}


class Types:
    """One of the reference's type tables (default_data or vinardo_data)."""

    def __init__(self, rows):
        self.rows = rows
        self.xs_radius = [r["xs_radius"] for r in rows]
        self.hyd = [r["xs_hydrophobe"] for r in rows]
        self.don = [r["xs_donor"] for r in rows]
        self.acc = [r["xs_acceptor"] for r in rows]
        self.solv = [r["ad_solvation"] for r in rows]
        self.vol = [r["ad_volume"] for r in rows]

    def by_name(self, name):
        """string_to_smina_type: two characters or fewer name an AD4 type
        (then the equivalences, then the generic metal), longer ones a smina
        type; None when unknown."""
        if len(name) <= 2:
            for k, r in enumerate(self.rows):
                if r["adname"] == name:
                    return k
            for a, b in REF["equivalences"]:
                if a == name:
                    return self.by_name(b)
            if name in REF["non_ad_metals"]:
                return [r["sm"] for r in self.rows].index("GenericMetal")
            return None
        for k, r in enumerate(self.rows):
            if r["smina_name"] == name:
                return k
        return None

    def hbond(self, a, b):
        return (self.don[a] and self.acc[b]) or (self.don[b] and self.acc[a])

    def anti_hbond(self, a, b):
        if self.don[a] and not self.acc[a]:
            return self.don[b] and not self.acc[b]
        if not self.don[a] and self.acc[a]:
            return not self.don[b] and self.acc[b]
        return False


def _exp(x):
    return np.array([math.exp(v) for v in np.asarray(x, np.float64).ravel()]).reshape(np.shape(x))


def _gaussian(x, width):
    return _exp(-((x / width) ** 2))


def _slope_step(bad, good, x):
    if bad < good:
        return np.where(x <= bad, 0.0, np.where(x >= good, 1.0, (x - bad) / (good - bad)))
    return np.where(x >= bad, 0.0, np.where(x <= good, 1.0, (x - bad) / (good - bad)))


def _int_pow(x, n):
    out = np.ones_like(x)
    for _ in range(n):
        out = out * x
    return out


def _vdw_coefficients(n, m, position, depth):
    c_n = _int_pow(np.float64(position), n) * depth * m / (float(n) - float(m))
    c_m = _int_pow(np.float64(position), m) * depth * n / (float(m) - float(n))
    return c_n, c_m


def _capped_inverse(t, cap):
    return np.where(t < EPS, cap, np.minimum(cap, 1.0 / np.where(t < EPS, 1.0, t)))


class Term:
    def __init__(self, desc, types):
        self.desc = desc
        self.kind = None
        for name, (pat, dep) in PATTERNS.items():
            m = re.fullmatch(pat, desc)
            if m:
                self.kind, self.dep = name, dep
                self.args = list(m.groups())
                break
        if self.kind is None:
            raise ValueError("unknown term " + desc)
        self.cutoff = float(self.args[-1])
        self.T = types
        if self.kind.startswith("atom_type_"):
            self.t1, self.t2 = types.by_name(self.args[0]), types.by_name(self.args[1])
            if self.t1 is None or self.t2 is None:
                raise ValueError("invalid atom type in " + desc)
        if self.kind in ("electrostatic", "atom_type_inverse_power"):
            p = float(self.args[0] if self.kind == "electrostatic" else self.args[2])
            if p not in (1.0, 2.0):
                raise ValueError("invalid exponent in " + desc)
        if self.kind == "vdw":
            if (float(self.args[0]), float(self.args[1])) not in ((4.0, 8.0), (6.0, 12.0)):
                raise ValueError("unsupported exponents in " + desc)

    def _opt(self, a, b):
        return self.T.xs_radius[a] + self.T.xs_radius[b]

    def eval(self, a, b, r):
        """charge-independent value at distances r for types (a, b)"""
        T, k, f = self.T, self.kind, [float(x) for x in self.args[:-1] if not re.fullmatch(r"[A-Za-z]\w*", x)]
        zero = np.zeros_like(r)
        if k == "gauss":
            return _gaussian(r - (self._opt(a, b) + f[0]), f[1])
        if k == "repulsion":
            d = r - (self._opt(a, b) + f[0])
            return np.where(d > 0, 0.0, d * d)
        if k in ("hydrophobic", "non_hydrophobic"):
            ok = (T.hyd[a] and T.hyd[b]) if k == "hydrophobic" else (not T.hyd[a] and not T.hyd[b])
            return _slope_step(f[1], f[0], r - self._opt(a, b)) if ok else zero
        if k == "non_dir_h_bond":
            return _slope_step(f[1], f[0], r - self._opt(a, b)) if T.hbond(a, b) else zero
        if k == "vdw":
            i, j, s, cap = int(f[0]), int(f[1]), f[2], f[3]
            d0 = self._opt(a, b)
            c_i, c_j = _vdw_coefficients(i, j, d0, 1.0)
            rr = np.where(r > d0 + s, r - s, np.where(r < d0 - s, r + s, d0))
            r_i, r_j = _int_pow(rr, i), _int_pow(rr, j)
            ok = (r_i > EPS) & (r_j > EPS)
            return np.where(ok, np.minimum(cap, c_i / np.where(ok, r_i, 1) + c_j / np.where(ok, r_j, 1)), cap)
        if k == "non_dir_h_bond_lj":
            if not T.hbond(a, b):
                return zero
            o, cap = f
            c_i, c_j = _vdw_coefficients(10, 12, self._opt(a, b) + o, 5.0)
            r_i, r_j = _int_pow(r, 10), _int_pow(r, 12)
            ok = (r_i > EPS) & (r_j > EPS)
            return np.where(ok, np.minimum(cap, c_i / np.where(ok, r_i, 1) + c_j / np.where(ok, r_j, 1)), cap)
        if k in ("non_dir_anti_h_bond_quadratic", "donor_donor_quadratic", "acceptor_acceptor_quadratic"):
            ok = (T.anti_hbond(a, b) if k == "non_dir_anti_h_bond_quadratic"
                  else (T.don[a] and T.don[b]) if k == "donor_donor_quadratic" else (T.acc[a] and T.acc[b]))
            if not ok:
                return zero
            d = r - (self._opt(a, b) + f[0])
            return np.where(d > 0, 0.0, d * d)
        match = (a == self.t1 and b == self.t2) or (a == self.t2 and b == self.t1) if k.startswith("atom_type_") else False
        if k == "atom_type_gaussian":
            return _gaussian(r - (self._opt(self.t1, self.t2) + f[0]), f[1]) if match else zero
        if k == "atom_type_linear":
            return _slope_step(f[1], f[0], r - self._opt(self.t1, self.t2)) if match else zero
        if k == "atom_type_quadratic":
            if not match:
                return zero
            d = r - (self._opt(self.t1, self.t2) + f[0])
            return np.where(d > 0, 0.0, d * d)
        if k == "atom_type_inverse_power":
            return _capped_inverse(_int_pow(r, int(f[0])), f[1]) if match else zero
        raise AssertionError(k)

    def eval_components(self, a, b, r):
        """charge-dependent terms: (type only, |q_a|, |q_b|, q_a q_b) components"""
        T, f = self.T, [float(x) for x in self.args[:-1]]
        out = [np.zeros_like(r) for _ in range(4)]
        if self.kind == "electrostatic":
            out[3] = _capped_inverse(_int_pow(r, int(f[0])), f[1])
            return out
        sigma, q = f
        df = _exp(-((r / (2 * sigma)) ** 2))
        out[0] = out[0] + T.solv[a] * T.vol[b] * df
        out[1] = out[1] + q * T.vol[b] * df
        out[0] = out[0] + T.solv[b] * T.vol[a] * df
        out[2] = out[2] + q * T.vol[a] * df
        return out


def scoring(terms_and_weights, vinardo=False):
    """(terms, weights) of the distance terms, in the order the reference
    keeps them: charge-independent terms in file order, then charge-dependent
    ones (weighted_terms.cpp:30-45)."""
    types = Types(REF["vinardo_types"] if vinardo else REF["types"])
    indep, dep = [], []
    for desc, w in terms_and_weights:
        if desc in CONF_INDEPENDENT:
            continue
        t = Term(desc, types)
        (dep if t.dep else indep).append((t, float(w)))
    return indep, dep


def parse_custom(text):
    """custom_terms::add_terms_from_file: 'weight term' per line, # comments"""
    out = []
    for line in text.splitlines():
        if not line or line.startswith("#"):
            continue
        parts = line.split()
        if len(parts) >= 2:
            out.append((parts[1], float(parts[0])))
    return out


def tables(terms_and_weights, factor=32.0, vinardo=False):
    """precalculate_linear: smooth [pair][i][c][e, dor] and fast [pair][i][c]"""
    indep, dep = scoring(terms_and_weights, vinardo)
    cutoff = max([t.cutoff for t, _ in indep + dep] + [0.0])
    nc = 4 if dep else 1
    cutoff_sqr = cutoff * cutoff
    n = int(factor * cutoff_sqr) + 3
    rs = np.sqrt(np.arange(n + 2, dtype=np.float64) / factor)
    smooth = np.zeros((NPAIRS, n, nc, 2))
    fast = np.zeros((NPAIRS, n, nc))
    r = rs[:n]
    for t2 in range(NT):
        for t1 in range(t2 + 1):
            p = t1 + t2 * (t2 + 1) // 2
            e = [np.zeros(n) for _ in range(nc)]
            for t, w in indep:
                e[0] = e[0] + w * t.eval(t1, t2, r)
            for t, w in dep:
                comp = t.eval_components(t1, t2, r)
                for c in range(4):
                    e[c] = e[c] + comp[c] * w
            for c in range(nc):
                E = e[c]
                smooth[p, :, c, 0] = E
                dor = np.zeros(n)
                dor[1:n - 1] = (E[2:] - E[:-2]) / ((rs[2:n] - rs[:n - 2]) * rs[1:n - 1])
                smooth[p, :, c, 1] = dor
                f2 = np.append(E[1:], 0.0)
                fast[p, :, c] = (f2 + E) / 2
    return smooth, fast
