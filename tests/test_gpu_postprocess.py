"""Static-analysis post-processing on the device: StaticAnalysis.AverageElementToNode against the oracle
(bit for bit: the device sums each node's elements in the reference's element order)."""
import numpy as np
import pytest

from mycel_b200 import api
from mycel_b200.model import ArgumentError, FeMaterial, FeModel, GridSpec
from models import carved_model

pytestmark = pytest.mark.gpu


def test_reference_case(ctx):
    g = GridSpec(2, 2, 1, 1.0)
    m = FeModel(g, np.ones(4, dtype=np.uint8), FeMaterial(1000.0, 0.3), [0, 1, 2, 3, 4, 5])
    out = api.StaticAnalysis.average_element_to_node(m, [10.0, 20.0, 30.0, 40.0], ctx=ctx)
    assert out[g.node_index(1, 1, 0)] == 25.0 and out[g.node_index(0, 0, 0)] == 10.0


@pytest.mark.parametrize("shape", [(5, 3, 2), (31, 12, 9), (40, 20, 10)])
def test_average_matches_oracle_on_carved_domains(oracle, ctx, shape):
    m = carved_model(*shape, seed=6, frac=0.25)
    es = np.random.default_rng(1).uniform(-3.0, 7.0, m.total_elements)
    ref = oracle.Model(m).average_element_to_node(es)
    out = api.StaticAnalysis.average_element_to_node(m, es, ctx=ctx)
    assert np.array_equal(out, ref)


def test_von_mises_nodal_field(oracle, ctx):
    """The App's use: element von Mises of a static solve, averaged to the nodes."""
    m = carved_model(24, 10, 8, seed=5)
    r = api.StaticAnalysis.run(m, ctx=ctx)
    out = api.StaticAnalysis.average_element_to_node(m, r.von_mises_per_element, ctx=ctx)
    assert np.array_equal(out, oracle.Model(m).average_element_to_node(r.von_mises_per_element))
    assert out.max() > 0


def test_wrong_length_is_an_argument_error(ctx):
    m = carved_model(6, 4, 3, seed=2)
    with pytest.raises(ArgumentError, match="elementScalar length must equal TotalElements"):
        api.StaticAnalysis.average_element_to_node(m, np.zeros(m.total_elements - 1), ctx=ctx)
