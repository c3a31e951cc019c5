"""Writes tests/golden/known_answers.json: the hand-literal known-answer cases of
the reference test suite for the SparsePauliVector path, transcribed as data
(the Pauli strings, coefficients, strategies and expected survivors/values of
test/test_truncation.jl, test/test_channels.jl and test/test_sparse_pauli_vector.jl).

Run: python tests/golden/make_known_answers.py
"""
import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))

cases = []


def trunc(name, src, terms, strategy, keep, corr=None, extra=None):
    c = {"kind": "truncate", "name": name, "source": src, "N": len(terms[0][0]),
         "terms": terms, "strategy": strategy, "keep": keep}
    if corr is not None:
        c["energy_delta"] = corr
    if extra:
        c.update(extra)
    cases.append(c)


trunc("CoeffTruncation", "test/test_truncation.jl:16-28",
      [["IIII", 1.0], ["XIII", 0.5], ["IXII", 1e-4], ["IIXI", 1e-8]],
      ["coeff", 1e-3], ["IIII", "XIII"])
trunc("WeightTruncation", "test/test_truncation.jl:30-44",
      [["IIII", 1.0], ["XIII", 0.5], ["XXII", 0.3], ["XXXI", 0.2], ["XXXX", 0.1]],
      ["weight", 2], ["IIII", "XIII", "XXII"])
trunc("XWeightTruncation", "test/test_truncation.jl:46-67",
      [["IIII", 1.0], ["ZZZZ", 0.9], ["XIII", 0.5], ["YZII", 0.4], ["XYII", 0.3], ["XYZX", 0.1]],
      ["xweight", 1], ["IIII", "ZZZZ", "XIII", "YZII"],
      extra={"x_weight": {"IIII": 0, "ZZZZ": 0, "YZII": 1, "XYZX": 3}})
trunc("XWeightDampedTruncation criterion", "test/test_truncation.jl:81-95",
      [["ZZZZ", 1.0], ["XIII", 0.01], ["XYII", 0.5], ["XYXI", 0.1], ["XYXY", 1.0]],
      ["xwdamped", 0.5, 0.05], ["ZZZZ", "XYII", "XYXY"], extra={"values": {"XYXY": 1.0}})
trunc("XWeightDamped composite == sequential", "test/test_truncation.jl:107-117",
      [["ZZZZ", 1.0], ["XYII", 0.5], ["XYXI", 0.4], ["XIII", 1e-8]],
      ["comp", [["xwdamped", 0.5, 0.05], ["xweight", 2]]], ["ZZZZ", "XYII"])
trunc("MajoranaWeightTruncation(0)", "test/test_truncation.jl:124-138",
      [["IIII", 1.0], ["XIII", 0.5], ["XXXX", 0.1]],
      ["majorana", 0], ["IIII"], extra={"majorana_weight": {"IIII": 0}})
trunc("WeightDampedTruncation criterion", "test/test_truncation.jl:153-167",
      [["IIII", 1.0], ["XIII", 0.01], ["XXII", 0.5], ["XXXI", 0.1], ["XXXX", 1.0]],
      ["wdamped", 0.5, 0.05], ["IIII", "XXII", "XXXX"], extra={"values": {"XXXX": 1.0}})
trunc("WeightDamped composite == sequential", "test/test_truncation.jl:179-189",
      [["IIII", 1.0], ["XXII", 0.5], ["XXXI", 0.4], ["XIII", 1e-8]],
      ["comp", [["wdamped", 0.5, 0.05], ["weight", 2]]], ["IIII", "XXII"])
trunc("WeightDamped with EnergyCorrection", "test/test_truncation.jl:192-200",
      [["IIII", 1.0], ["ZZZZ", 0.1]], ["wdamped", 1.0, 0.05], ["IIII"], corr=-0.1)
trunc("CompositeTruncation", "test/test_truncation.jl:250-275",
      [["IIII", 1.0], ["XIII", 0.5], ["XXXI", 0.3], ["IIXI", 1e-8]],
      ["comp", [["coeff", 1e-3], ["weight", 2]]], ["IIII", "XIII"])
trunc("NoCorrection", "test/test_truncation.jl:277-286",
      [["IIII", 1.0], ["XIII", 1e-8]], ["coeff", 1e-3], ["IIII"])
trunc("EnergyCorrection", "test/test_truncation.jl:288-303",
      [["IIII", 1.0], ["ZIII", 0.5], ["XIII", 0.01]], ["coeff", 0.1], ["IIII", "ZIII"], corr=0.0)


def chan(name, src, kind, prm, terms, expect):
    cases.append({"kind": "channel", "name": name, "source": src, "N": len(terms[0][0]),
                  "channel": kind, "prm": prm, "terms": terms, "expect": expect})


p = 0.1
ld = 1 - 4 * p / 3
chan("depolarizing closed form", "test/test_channels.jl:123-133", "depolarizing", [p],
     [["XIZ", 1.0], ["YYY", 2.0], ["III", 7.0]], {"XIZ": ld ** 2, "YYY": 2.0 * ld ** 3, "III": 7.0})
lam = 1 - 2 * 0.2
chan("dephasing closed form", "test/test_channels.jl:135-145", "dephasing", [0.2],
     [["XIZ", 1.0], ["YYZ", 1.0], ["ZIZ", 1.0]], {"XIZ": lam, "YYZ": lam ** 2, "ZIZ": 1.0})
lam = 1 - 2 * 0.3
chan("bit-flip closed form", "test/test_channels.jl:147-157", "bit_flip", [0.3],
     [["XIZ", 1.0], ["YYZ", 1.0], ["XIX", 1.0]], {"XIZ": lam, "YYZ": lam ** 3, "XIX": 1.0})
lam = 1 - 2 * 0.25
chan("bit-phase-flip closed form", "test/test_channels.jl:159-169", "bit_phase_flip", [0.25],
     [["XIZ", 1.0], ["YYY", 1.0], ["XYZ", 1.0]], {"XIZ": lam ** 2, "YYY": 1.0, "XYZ": lam ** 2})
pX, pY, pZ = 0.05, 0.10, 0.15
lX, lY, lZ = 1 - 2 * (pY + pZ), 1 - 2 * (pX + pZ), 1 - 2 * (pX + pY)
chan("pauli channel closed form", "test/test_channels.jl:171-179", "pauli", [pX, pY, pZ],
     [["XYZ", 1.0], ["XIX", 1.0]], {"XYZ": lX * lY * lZ, "XIX": lX * lX})

errors = [
    ["depolarizing", [-0.1], None], ["depolarizing", [1.1], None], ["dephasing", [-0.1], None],
    ["bit_flip", [2.0], None], ["bit_phase_flip", [-1.0], None],
    ["pauli", [-0.1, 0.1, 0.1], None], ["pauli", [0.5, 0.5, 0.5], None],
    ["depolarizing", [0.1], [0]], ["depolarizing", [0.1], [4]], ["pauli", [0.1, 0.1, 0.1], 4],
]
cases.append({"kind": "channel_errors", "name": "argument validation", "source": "test/test_channels.jl:286-305",
              "N": 3, "terms": [["XIZ", 1.0]], "errors": errors})
cases.append({"kind": "word_type", "name": "word type selection", "source": "test/test_sparse_pauli_vector.jl:10-22",
              "nwords": {"1": 1, "64": 1, "65": 2, "128": 2}, "error": [129]})
cases.append({"kind": "weight_decay", "name": "depolarizing_p_for_weight_decay edge cases",
              "source": "test/test_channels.jl:360-368",
              "values": [[0.0, 1.0, 0.0], [1.0, 0.0, 0.0], [0.7, 0.4, 0.75 * (1 - math.exp(-0.28))]]})

with open(os.path.join(HERE, "known_answers.json"), "w") as f:
    json.dump({"generator": "tests/golden/make_known_answers.py", "cases": cases}, f, indent=1)
print(len(cases), "cases")
