"""Output-step selection (OutputSelection::parse, src/output/output_variables.hpp:
27-70): the library's parser against the reference's own parser (compiled
from the reference tree, oracle/_ref) on hand-written and random
specifications, errors included."""

import numpy as np
import pytest

from grt import lib
from grt.lib import GrtError, OUTPUT_FIELDS

SPECS = [
    "all", "id", "id,frequency,x0,x1,x2,x3,k0,k1,k2,k3,I,Q,U,V,phase", " x0 , x1 ", "[x0, x1]",
    '["id", "x0", "terminate"]', "['phase', 'I']", "x0,x0,x0", "I,all", "all,foo", "x0,,x1", ",x0", "x0,",
    "[ ]", "", "   ", ",", "foo", "x0, bar", "X0", '"x0', "id,\"phi_disp\",'theta_disp',dlambda",
    "terminate,phase,emission_frame_energy", "[all]", "['all']", "[x0", "x0]", " [ id , k3 ] ",
]


def ours(spec):
    try:
        return [OUTPUT_FIELDS.index(n) for n in lib.parse_output_variables(spec)], None
    except GrtError as e:
        return None, str(e).split(": ", 1)[1]


def theirs(reference, spec):
    try:
        return reference.parse_output_variables(spec), None
    except ValueError as e:
        return None, str(e)


def random_specs(n, seed=5):
    rng = np.random.default_rng(seed)
    tokens = list(OUTPUT_FIELDS) + ["all", "", " ", "foo", '"x0"', "'I'", "[", "]", " id "]
    out = []
    for _ in range(n):
        k = int(rng.integers(1, 6))
        parts = [tokens[int(rng.integers(len(tokens)))] for _ in range(k)]
        s = ",".join(parts)
        if rng.random() < 0.3:
            s = "[" + s + "]"
        out.append(s)
    return out


@pytest.mark.parametrize("spec", SPECS)
def test_selection_matches_reference(reference, spec):
    assert ours(spec) == theirs(reference, spec)


def test_random_selections_match_reference(reference):
    for spec in random_specs(400):
        assert ours(spec) == theirs(reference, spec), spec
