"""Input decks in the reference's ParmParse format.

The reference reads its parameters with AMReX ParmParse: lines
``prefix.key = token token ...`` ('#' starts a comment, double quotes group
a token, a later line overrides an earlier one for the same key), numeric
tokens through the AMReX expression parser with the deck's
``my_constants.*`` (queryWithParser / queryArrWithParser).  The NEGF keys of
one nanostructure are read twice, first from ``NS_default`` and then from
the structure's own name, so the name's values win
(Read_NanostructureProperties, Source/Solver/Transport/NEGF/
NEGF_Common.cpp:699-718); the CNT keys the same way from ``CNT_default``
(CNT.cpp:43-59).  The transport loop reads ``transport.*``
(Transport.cpp:56-267).

Deck -> engine:
    deck = Deck.from_file(path)
    for name in deck.transport()["NS_names"]:
        tube = CNT(**deck.tube_kwargs(name))

BLOCK_SIZE (the number of modes) is a compile-time constant of the
reference; here it is the key ``num_modes`` of the structure (or of
NS_default), default 1.  ``precision`` (fp64 | mixed) selects the engine's
precision mode.  Keys of the mesh, embedded boundaries, plotting and the
electrostatics are read by the reference's other layers and are ignored
here.
"""
from __future__ import annotations

import ast
import math
import operator
import shlex

_FUNCS = {
    "sqrt": math.sqrt, "exp": math.exp, "log": math.log, "log10": math.log10, "sin": math.sin, "cos": math.cos,
    "tan": math.tan, "asin": math.asin, "acos": math.acos, "atan": math.atan, "atan2": math.atan2,
    "sinh": math.sinh, "cosh": math.cosh, "tanh": math.tanh, "abs": abs, "fabs": abs, "floor": math.floor,
    "ceil": math.ceil, "min": min, "max": max, "pow": math.pow,
}
_BIN = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv,
        ast.Pow: operator.pow, ast.Mod: math.fmod}
_UN = {ast.UAdd: operator.pos, ast.USub: operator.neg}


class DeckError(ValueError):
    pass


class Deck:
    """The key/value table of a deck and its expression evaluator."""

    def __init__(self, text: str = ""):
        self.table: dict[str, list[str]] = {}
        self._const_cache: dict[str, float] = {}
        self._busy: set[str] = set()
        for lineno, raw in enumerate(text.splitlines(), 1):
            line = raw.split("#", 1)[0].strip() if '"' not in raw else self._strip_comment(raw)
            if not line:
                continue
            if "=" not in line:
                raise DeckError(f"line {lineno}: expected 'key = value': {raw.strip()!r}")
            key, val = line.split("=", 1)
            key = key.strip()
            try:
                toks = shlex.split(val, posix=True)
            except ValueError as e:
                raise DeckError(f"line {lineno}: {e}") from None
            self.table[key] = toks

    @staticmethod
    def _strip_comment(raw: str) -> str:
        out, quoted = [], False
        for ch in raw:
            if ch == '"':
                quoted = not quoted
            if ch == "#" and not quoted:
                break
            out.append(ch)
        return "".join(out).strip()

    @classmethod
    def from_file(cls, path: str) -> "Deck":
        with open(path) as f:
            return cls(f.read())

    # ------------------------------------------------------------------ expressions
    def constant(self, name: str) -> float:
        if name in self._const_cache:
            return self._const_cache[name]
        key = "my_constants." + name
        if key not in self.table:
            if name == "pi":
                return math.pi
            raise DeckError(f"unknown symbol {name!r}")
        if name in self._busy:
            raise DeckError(f"my_constants.{name} refers to itself")
        self._busy.add(name)
        try:
            v = self.eval(" ".join(self.table[key]))
        finally:
            self._busy.discard(name)
        self._const_cache[name] = v
        return v

    def eval(self, expr: str) -> float:
        """Value of an arithmetic expression of numbers, my_constants, pi and
        the parser's functions ('^' and '**' are powers)."""
        try:
            tree = ast.parse(expr.replace("^", "**"), mode="eval")
        except SyntaxError:
            raise DeckError(f"cannot parse {expr!r}") from None
        return float(self._ev(tree.body))

    def _ev(self, n):
        if isinstance(n, ast.Constant) and isinstance(n.value, (int, float)):
            return n.value
        if isinstance(n, ast.BinOp) and type(n.op) in _BIN:
            return _BIN[type(n.op)](self._ev(n.left), self._ev(n.right))
        if isinstance(n, ast.UnaryOp) and type(n.op) in _UN:
            return _UN[type(n.op)](self._ev(n.operand))
        if isinstance(n, ast.Name):
            return self.constant(n.id)
        if isinstance(n, ast.Call) and isinstance(n.func, ast.Name) and n.func.id in _FUNCS and not n.keywords:
            return _FUNCS[n.func.id](*[self._ev(a) for a in n.args])
        raise DeckError(f"unsupported expression element {ast.dump(n)[:60]}")

    # ------------------------------------------------------------------ queries
    def has(self, prefix: str, name: str) -> bool:
        return f"{prefix}.{name}" in self.table

    def query_str(self, prefix, name, default=None):
        v = self.table.get(f"{prefix}.{name}")
        return default if v is None else " ".join(v)

    def query_strs(self, prefix, name, default=None):
        v = self.table.get(f"{prefix}.{name}")
        return default if v is None else list(v)

    def query(self, prefix, name, default=None, kind=float):
        """queryWithParser: one value (int values must be integral)."""
        v = self.table.get(f"{prefix}.{name}")
        if v is None:
            return default
        x = self.eval(" ".join(v))
        return self._kind(x, kind, prefix, name)

    def query_arr(self, prefix, name, n=None, default=None, kind=float):
        """queryArrWithParser: one expression per token (n of them when given)."""
        v = self.table.get(f"{prefix}.{name}")
        if v is None:
            return default
        vals = [self._kind(self.eval(t), kind, prefix, name) for t in v]
        if n is not None and len(vals) < n:
            raise DeckError(f"{prefix}.{name} needs {n} values, has {len(vals)}")
        return vals[:n] if n is not None else vals

    @staticmethod
    def _kind(x, kind, prefix, name):
        if kind is int:
            if abs(x - round(x)) > 1e-9:
                raise DeckError(f"{prefix}.{name} must be an integer, got {x}")
            return int(round(x))
        return kind(x)

    def _layered(self, defaults: str, name: str, key: str, getter):
        """Value from `name` if given there, else from the defaults namespace."""
        v = getter(name, key)
        return v if v is not None else getter(defaults, key)

    # ------------------------------------------------------------------ the engine's parameters
    def transport(self) -> dict:
        """transport.* keys of the self-consistent loop (Transport.cpp:56-267)."""
        p = "transport"
        names = self.query_strs(p, "NS_names")
        if names is None and self.has(p, "NS_num"):
            names = [f"NS{i}" for i in range(self.query(p, "NS_num", kind=int))]
        return dict(NS_names=names or [],
                    Broyden_fraction=self.query(p, "Broyden_fraction", 0.1),
                    Broyden_max_norm=self.query(p, "Broyden_max_norm", 1e-5),
                    Broyden_norm_type=self.query_str(p, "Broyden_norm_type", "relative"),
                    Broyden_threshold_maxstep=self.query(p, "Broyden_threshold_maxstep", 200, kind=int),
                    reset_with_previous_charge_distribution=self.query(
                        p, "reset_with_previous_charge_distribution", 0, kind=int),
                    NS_initial_deposit_value=self.query(p, "NS_initial_deposit_value", 0.0))

    def tube_kwargs(self, name: str, num_modes: int | None = None) -> dict:
        """Keyword arguments of negf.CNT for the nanostructure `name`: NEGF keys
        from NS_default then `name` (NEGF_Common.cpp:375-643), CNT keys from
        CNT_default then `name` (CNT.cpp:13-21, 43-59)."""
        def num(key, kind=float):
            return self._layered("NS_default", name, key, lambda p, k: self.query(p, k, kind=kind))

        def arr(key, n=None, kind=float):
            return self._layered("NS_default", name, key, lambda p, k: self.query_arr(p, k, n, kind=kind))

        def cnt(key, n=None, kind=float):
            if n is None:
                return self._layered("CNT_default", name, key, lambda p, k: self.query(p, k, kind=kind))
            return self._layered("CNT_default", name, key, lambda p, k: self.query_arr(p, k, n, kind=kind))

        kw = {}
        tid = cnt("type_id", 2, int)
        if tid is not None:
            kw["type_id"] = tuple(tid)
        for key in ("acc", "gamma"):
            v = cnt(key)
            if v is not None:
                kw[key] = v
        v = num("num_unitcells", int)
        if v is not None:
            kw["num_unitcells"] = v
        modes = num_modes if num_modes is not None else num("num_modes", int)
        kw["num_modes"] = modes if modes is not None else 1
        # contacts (Read_TerminalParams, NEGF_Common.cpp:375-432): explicit contact_mu when
        # contact_mu_specified, else both contacts at contact_Fermi_level (no terminal bias)
        if num("contact_mu_specified", int):
            mu = arr("contact_mu", 2)
            if mu is not None:
                kw["contact_mu"] = tuple(mu)
        else:
            ef = num("contact_Fermi_level")
            if ef is not None:
                kw["contact_mu"] = (ef, ef)
        for key, n, kind in (("contact_T", 2, float), ("eq_integration_pts", 3, int),
                             ("Fermi_tail_factors", 2, float), ("kT_window_around_singularity", 2, float)):
            v = arr(key, n, kind)
            if v is not None:
                kw[key] = tuple(v)
        npaths = num("num_noneq_paths", int)
        ne = arr("noneq_integration_pts", npaths, int)
        if ne is not None:
            kw["noneq_integration_pts"] = tuple(ne)
        if npaths is not None and npaths > 1:
            cuts = arr("noneq_percent_intercuts", npaths - 1)
            if cuts is not None:
                kw["noneq_percent_intercuts"] = tuple(cuts)
        dens = arr("noneq_integration_pts_density", npaths)
        if dens is not None:
            kw["noneq_integration_pts_density"] = tuple(dens)
        for key in ("E_valence_min", "E_pole_max", "E_zPlus_imag"):
            v = num(key)
            if v is not None:
                kw[key] = v
        for key in ("use_decimation", "decimation_max_iter", "decimation_layers", "flatband_dos_integration_pts",
                    "flag_adaptive_integration_limits", "integrand_correction_interval"):
            v = num(key, int)
            if v is not None:
                kw[key] = v
        prec = self._layered("NS_default", name, "precision", lambda p, k: self.query_str(p, k))
        if prec is not None:
            kw["precision"] = prec
        return kw
