"""Extract the reference's known answers for the partition metrics into evaluate_known_answers.json.

Reads test/evaluate_test.cpp of the reference as text (it is not compiled or run here): two
contingency tables with their vertex counts and the expected F1 score (and, for the first, the
Rand index, precision and recall).
Run:  python tests/golden/make_evaluate_fixture.py /path/to/reference  (or set SBP_REFERENCE_DIR)
"""
import json
import os
import re
import sys


def table(text, name):
    body = text[text.index(name + " = {"):]
    body = body[:body.index("};")]
    return [[int(x) for x in re.findall(r"\d+", row)] for row in re.findall(r"\{([^{}]*)\}", body)]


def main(ref):
    src = open(os.path.join(ref, "test/evaluate_test.cpp")).read()
    num = lambda name: float(re.search(name + r" = ([0-9.]+);", src).group(1))
    fixture = {
        "source": "reference test/evaluate_test.cpp",
        "matrix": table(src, "Matrix"), "num_vertices": int(num("N")),
        "rand_index": num("RandIndex"), "precision": num("Precision"), "recall": num("Recall"), "f1": num("F1"),
        "matrix2": table(src, "Matrix2"), "num_vertices2": int(num("N2")), "f1_2": num("F12"),
    }
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "evaluate_known_answers.json")
    with open(out, "w") as f:
        json.dump(fixture, f)
    print(out)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SBP_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: make_evaluate_fixture.py <reference checkout> (or set SBP_REFERENCE_DIR)")
    main(ref)
