"""Output-step selection (OutputSelection::parse, src/output/output_variables.hpp:
27-70) and the output keys of the TOML config (toml_config.hpp:225-243): the
library's parser against the reference's own parser (compiled from the
reference tree, oracle/_ref) on hand-written and random specifications,
errors included."""

import numpy as np
import pytest

from grt import config, lib, workloads
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


def test_output_options_from_toml(tmp_path):
    p = workloads.C1.params()
    text = config.toml_text(p, str(tmp_path / "np"), str(tmp_path / "out"), "run")
    path = tmp_path / "c.toml"
    path.write_text(text)
    spec, stride = lib.output_options_from_toml(path)
    assert lib.parse_output_variables(spec) == ["id", "frequency", "x0", "x1", "x2", "x3", "k0", "k1", "k2", "k3",
                                                "I", "Q", "U", "V", "terminate", "phase"]
    assert stride == 1
    path.write_text(text.replace("stride = 1", "stride = 7").replace(
        'variables = ["id"', 'variables = ["dlambda", "id"'))
    spec, stride = lib.output_options_from_toml(path)
    assert stride == 7 and lib.parse_output_variables(spec)[:2] == ["dlambda", "id"]
    # defaults when the keys are absent
    path.write_text("\n".join(l for l in text.splitlines() if not l.startswith(("stride", "variables"))) + "\n")
    spec, stride = lib.output_options_from_toml(path)
    assert stride == 1 and spec == lib.DEFAULT_OUTPUT_VARIABLES
    for bad, msg in (("stride = 0", "output.stride must be positive"),
                     ('variables = "x0, nope"', "unknown output variable: nope")):
        lines = [l for l in text.splitlines() if not l.startswith(("stride", "variables"))]
        lines.insert(lines.index("[output]") + 1, bad)
        path.write_text("\n".join(lines) + "\n")
        with pytest.raises(GrtError, match=msg):
            lib.output_options_from_toml(path)
