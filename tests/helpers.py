"""Shared test helpers: molecules, basis loading, the product package."""
import importlib
import json
import os

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")

WATER = [["O", 0.0, 0.0, 0.1173], ["H", 0.0, 0.7572, -0.4692], ["H", 0.0, -0.7572, -0.4692]]


def pfk():
    """The product package (its directory name is not an identifier)."""
    return importlib.import_module("planck-refactored_b200")


def basis_library():
    return pfk().basis.load_library()


def regression_cases():
    with open(os.path.join(GOLDEN, "regression_cases.json")) as f:
        return {c["id"]: c for c in json.load(f)["cases"]}


def water_cluster(*a, **k):
    return pfk().workloads.water_cluster(*a, **k)


def alkane(*a, **k):
    return pfk().workloads.alkane(*a, **k)


def random_shells(*a, **k):
    return pfk().workloads.random_shells(*a, **k)


def onee_highprec():
    """40-digit nuclear-attraction matrix of the random s..f test basis
    (tests/golden/make_onee_highprec.py): {"V": nb x nb, "coords": nuclei}."""
    with open(os.path.join(GOLDEN, "onee_highprec.json")) as f:
        g = json.load(f)
    nb = g["nbasis"]
    V = np.zeros((nb, nb))
    for i, j, v in g["V_upper"]:
        V[i, j] = V[j, i] = float(v)
    return {"V": V, "coords": np.array(g["nuclei"]["coords_bohr"])}


def random_density(nb, seed=5, scale=0.3):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(nb, nb)) * scale
    return A + A.T
