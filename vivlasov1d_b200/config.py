"""Run configuration: reads the reference's .cfg files.

The reference validates .cfg files with configobj against ``runspec.cfg``
(vlasov/core/config.py:15-31).  configobj is not available here, so this is
a small reader of the same INI dialect (``[section]``, ``key = value``,
``#`` comments, optional quotes) that fills in the same defaults and exposes
the same predicates (config.py:50-167).
"""
from __future__ import annotations


# section -> key -> (type, default); the defaults of runspec.cfg
RUNSPEC = {
    "grid": {
        "nt": (int, 100), "nx": (int, 128), "nv": (int, 256), "ht": (float, 0.1),
        "L": (float, 0.0), "vmin": (float, None), "vmax": (float, 5.0),
    },
    "solver": {
        "method": (str, "iterative"), "type": (str, "nonlinear"), "mode": (str, "split"),
        "timestepping": (str, "mp"), "poisson_bracket": (str, "ArakawaJ4"),
        "laplace_operator": (str, "CFD4"), "averaging_operator": (str, None),
        "dissipation_type": (str, None), "collision_operator": (str, None),
        "bracket_operator": (str, None), "preconditioner_type": (str, None),
        "preconditioner_scheme": (str, None), "initial_guess": (str, None),
        "lu_package": (str, "mumps"), "initial_iter": (int, 1),
        "petsc_ksp_rtol": (float, 1e-4), "petsc_ksp_atol": (float, 1e-50),
        "petsc_ksp_max_iter": (int, 1000), "petsc_snes_atol": (float, 1e-10),
        "petsc_snes_rtol": (float, 1e-14), "petsc_snes_stol": (float, 1e-16),
        "petsc_snes_max_iter": (int, 20), "coll_freq": (float, 0.0), "coll_diff": (float, 1.0),
        "coll_drag": (float, 1.0), "regularisation": (float, 0.0),
    },
    "initial_data": {
        "mass": (float, 1.0), "charge": (float, 1.0), "density": (float, 1.0),
        "temperature": (float, 1.0), "distribution_file": (str, None), "density_file": (str, None),
        "temperature_file": (str, None), "potential_file": (str, None),
        "distribution_python": (str, None), "density_python": (str, None),
        "temperature_python": (str, None), "potential_python": (str, None),
        "external_python": (str, None), "nfourier": (int, 0),
    },
    "io": {
        "output_dir": (str, "."), "nsave": (int, 1), "hdf5_input": (str, None),
        "hdf5_output": (str, None),
    },
}


def _convert(typ, raw):
    s = raw.strip()
    if len(s) >= 2 and s[0] == s[-1] and s[0] in "'\"":
        s = s[1:-1]
    elif s.endswith('"') and s.count('"') == 1:   # tolerate a stray closing quote
        s = s[:-1]
    if s in ("None", ""):
        return None
    if typ is int:
        return int(float(s))
    if typ is float:
        return float(s)
    return s


class Config(dict):
    """Dict of sections with the reference's accessor predicates."""

    def __init__(self, infile=None, text=None, overrides=None):
        super().__init__()
        for sec, keys in RUNSPEC.items():
            self[sec] = {k: d for k, (t, d) in keys.items()}
        if infile is not None:
            with open(infile) as fh:
                text = fh.read()
        if text is not None:
            self._parse(text)
        if overrides:
            for sec, kv in overrides.items():
                self[sec].update(kv)

    def _parse(self, text):
        section = None
        for line in text.splitlines():
            s = line.split("#", 1)[0].strip() if not line.strip().startswith("#") else ""
            if not s:
                continue
            if s.startswith("[") and s.endswith("]"):
                section = s[1:-1].strip()
                self.setdefault(section, {})
                continue
            if "=" not in s or section is None:
                continue
            k, v = s.split("=", 1)
            k = k.strip()
            spec = RUNSPEC.get(section, {}).get(k)
            typ = spec[0] if spec else str
            self[section][k] = _convert(typ, v)

    # predicates (config.py:50-167)
    def get_timestepping(self):
        return self["solver"]["timestepping"].lower()

    def get_poisson_bracket(self):
        return self["solver"]["poisson_bracket"].lower()

    def get_laplace_operator(self):
        return self["solver"]["laplace_operator"].lower()

    def is_averaging_operator_none(self):
        a = self["solver"]["averaging_operator"]
        return a is None or a.lower() == "none"

    def get_averaging_operator(self):
        return "point" if self.is_averaging_operator_none() else self["solver"]["averaging_operator"].lower()

    def is_preconditioner_none(self):
        t, s = self["solver"]["preconditioner_type"], self["solver"]["preconditioner_scheme"]
        return t is None or t.lower() == "none" or s is None or s.lower() == "none"

    def get_preconditioner(self):
        return "" if self.is_preconditioner_none() else self["solver"]["preconditioner_scheme"].lower()

    def is_dissipation_none(self):
        d = self["solver"]["dissipation_type"]
        return d is None or self["solver"]["coll_freq"] == 0. or d.lower() == "none"

    def is_dissipation_collisions(self):        # config.py:135-139
        d = self["solver"]["dissipation_type"]
        return not (d is None or self["solver"]["coll_freq"] == 0.) and d.lower() == "collisions"

    def is_dissipation_double_bracket(self):    # config.py:141-145
        d = self["solver"]["dissipation_type"]
        return not (d is None or self["solver"]["coll_freq"] == 0.) and d.lower() == "double_bracket"

    def get_collision_operator(self):           # config.py:148-154
        if not self.is_dissipation_collisions():
            return ""
        return (self["solver"]["collision_operator"] or "").lower()

    def get_double_bracket(self):               # config.py:156-162
        if not self.is_dissipation_double_bracket():
            return ""
        return (self["solver"]["bracket_operator"] or "").lower()
