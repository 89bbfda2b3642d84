"""Label -> einsum subscript mapping (contraction/contractor.py:48-144) of
the host layer against the oracle's restatement, with the reference's error
texts.  The mapping reads only the legs' labels, so plain stand-ins carry
them here (no device tensors)."""

from types import SimpleNamespace

import pytest

from oracle.blocksparse import labels_to_subscripts as o_labels
from tenax_b200.contraction import _labels_to_subscripts


def _pair(*label_lists):
    """Device-style stand-ins (``.indices``) and oracle-style ones (``.legs``)."""
    dev = [SimpleNamespace(indices=[SimpleNamespace(label=l) for l in ls]) for ls in label_lists]
    ora = [SimpleNamespace(legs=[SimpleNamespace(label=l) for l in ls]) for ls in label_lists]
    return dev, ora


CASES = [
    (["i", "j"], ["j", "k"]),                       # matrix product
    (["a", "b", "c"], ["c", "d"], ["d", "e"]),       # chain of three
    ([10, 2, "a"], ["B", 10]),                      # mixed int / str labels, sorted by str
    (["x", "y"], ["z"]),                            # outer product, nothing contracted
    (["p", "q", "r"], ["r", "q", "p"]),             # everything contracted: scalar
]


@pytest.mark.parametrize("labels", CASES)
def test_mapping_matches_oracle(labels):
    dev, ora = _pair(*labels)
    subs, out = _labels_to_subscripts(dev)
    o_subs, o_out = o_labels(ora)
    assert subs == o_subs
    assert [i.label for i in out] == [l.label for l in o_out]


def test_sort_order_and_free_label_order():
    dev, _ = _pair([10, 2, "a"], ["B", 10])
    subs, out = _labels_to_subscripts(dev)
    # str order: "10" < "2" < "B" < "a" -> a, b, c, d; free labels in first-appearance order
    assert subs == "abd,ca->bdc"
    assert [i.label for i in out] == [2, "a", "B"]


def test_explicit_output_labels():
    dev, ora = _pair(["i", "j"], ["j", "k"])
    subs, out = _labels_to_subscripts(dev, ["k", "i"])
    assert subs == o_labels(ora, ["k", "i"])[0] == "ab,bc->ca"


def test_errors_carry_the_reference_text():
    dev, _ = _pair(["i", "j"], ["j", "k"], ["j"])
    with pytest.raises(ValueError, match=r"Label 'j' appears 3 times across tensors\. Labels must appear at most 2 "
                                         r"times \(one per tensor to contract\)\."):
        _labels_to_subscripts(dev)
    dev, _ = _pair([f"l{i}" for i in range(53)])
    with pytest.raises(ValueError, match=r"Too many unique labels \(53\) for einsum encoding\. Maximum supported is "
                                         r"52 \(a-z \+ A-Z\)\."):
        _labels_to_subscripts(dev)
    dev, _ = _pair(["i", "j"], ["j", "k"])
    with pytest.raises(ValueError, match=r"output_labels contains 'j' which is not a free label\. Free labels are: "
                                         r"\['i', 'k'\]"):
        _labels_to_subscripts(dev, ["j"])
    dev, _ = _pair([f"l{i}" for i in range(52)])
    subs, _ = _labels_to_subscripts(dev)  # exactly 52 labels fit
    assert len(subs.split("->")[0]) == 52
