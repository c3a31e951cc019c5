"""Pins the CPU oracle (and the host strategy compiler) to the reference's
hand-literal known-answer tests, transcribed in tests/golden/known_answers.json."""
import json
import math
import os

import pytest

import orc
import pauliprop as pp
from helpers import CHANNEL_KIND, filt, key_of, strategy

CASES = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))["cases"]


def _oracle(case):
    N = case["N"]
    terms = [(*key_of(s), c) for s, c in case["terms"]]
    return orc.OracleSPV.from_terms(N, terms)


def _apply(v, spec):
    # truncate! applies composites strategy by strategy (truncation.jl:237-243)
    if spec[0] == "comp":
        for s in spec[1]:
            _apply(v, s)
    else:
        v.compact(filt(spec))


@pytest.mark.parametrize("case", [c for c in CASES if c["kind"] == "truncate"], ids=lambda c: c["name"])
def test_truncate_known_answer(case):
    v = _oracle(case)
    before = v.expect(0)
    _apply(v, case["strategy"])
    got = v.terms()
    assert set(got) == {key_of(s) for s in case["keep"]}
    for s, val in case.get("values", {}).items():
        assert got[key_of(s)] == val
    if "energy_delta" in case:
        assert v.expect(0) - before == pytest.approx(case["energy_delta"], abs=1e-15)
    # the composite strategy compiles to one MergeFilter with the same decision
    v2 = _oracle(case)
    v2.compact(filt(case["strategy"]))
    assert set(v2.terms()) == set(got)
    assert v.check()


def test_weight_helpers_known_answers():
    c = next(c for c in CASES if c["name"] == "XWeightTruncation")
    for s, w in c["x_weight"].items():
        b = pp.PauliBasis.from_string(s)
        assert pp.x_weight(b.z, b.x) == w
    assert pp.majorana_weight(4, 0, 0) == 0


@pytest.mark.parametrize("case", [c for c in CASES if c["kind"] == "channel"], ids=lambda c: c["name"])
def test_channel_closed_form(case):
    v = _oracle(case)
    v.channel(CHANNEL_KIND[case["channel"]], case["prm"])
    got = v.terms()
    for s, val in case["expect"].items():
        assert got[key_of(s)] == pytest.approx(val, rel=1e-14, abs=0)


def test_channel_argument_validation():
    case = next(c for c in CASES if c["kind"] == "channel_errors")
    N = case["N"]
    for kind, prm, qubits in case["errors"]:
        v = _oracle(case)
        if qubits is not None:
            with pytest.raises(pp.ArgumentError):
                pp.qubit_mask(N, qubits)
            continue
        with pytest.raises(orc.OracleError) as e:
            v.channel(CHANNEL_KIND[kind], prm)
        assert e.value.code == 1  # ArgumentError


def test_word_type_selection():
    case = next(c for c in CASES if c["kind"] == "word_type")
    for N, nw in case["nwords"].items():
        assert pp.nwords(int(N)) == nw
    for N in case["error"]:
        with pytest.raises(pp.PauliPropError):
            pp.nwords(N)


def test_weight_decay_p():
    case = next(c for c in CASES if c["kind"] == "weight_decay")
    for rate, dt, p in case["values"]:
        assert pp.depolarizing_p_for_weight_decay(rate, dt) == pytest.approx(p, abs=1e-15)


def test_pack_unpack_roundtrip_sign_bit():
    # test_sparse_pauli_vector.jl:24-38: N=128 with all 128 bits set
    allbits = (1 << 128) - 1
    z, x = pp.pack_keys(128, [(allbits, allbits), (1 << 127, 5)])
    assert z.shape == (2, 2) and int(z[0, 0]) == 2**64 - 1 and int(z[0, 1]) == 2**64 - 1
    assert pp.unpack_keys(z, x) == [(allbits, allbits), (1 << 127, 5)]
    v = orc.OracleSPV.from_terms(128, [(allbits, allbits, 1.0), (1 << 127, 5, 2.0), (3, 0, -1.0)])
    t = v.terms()
    assert t[(allbits, allbits)] == 1.0 and t[(1 << 127, 5)] == 2.0
    assert v.check()


def test_identity_term_invariant():
    # test_channels.jl:88-115 (unitality): the identity term is never scaled
    for kind in range(5):
        for p in (0.0, 0.1, 0.4, 0.7, 1.0):
            prm = [p / 3, p / 3, p / 3] if kind == 4 else [p]
            v = orc.OracleSPV.from_terms(4, [(0, 0, 3.14), (5, 3, 0.5)])
            v.channel(kind, prm)
            assert v.terms()[(0, 0)] == 3.14
