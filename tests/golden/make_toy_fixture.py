"""Extract the reference's known-answer values for the toy graphs into toy_example.json.

Reads the reference's GoogleTest sources as text (they are not compiled or run here):
  test/toy_example.hpp    edge list, assignments, ENTROPY, new-degree fixtures
  test/entropy_test.cpp   null-model MDL constants
  test/blockmodel_test.cpp, test/common_test.cpp, test/finetune_test.cpp, test/block_merge_test.cpp
                          expected degrees and Delta entries
Run:  python tests/golden/make_toy_fixture.py /path/to/reference
"""
import json
import os
import re
import sys


def main(ref):
    toy = open(os.path.join(ref, "test/toy_example.hpp")).read()
    ent = open(os.path.join(ref, "test/entropy_test.cpp")).read()
    bmt = open(os.path.join(ref, "test/blockmodel_test.cpp")).read()
    ftt = open(os.path.join(ref, "test/finetune_test.cpp")).read()
    bmg = open(os.path.join(ref, "test/block_merge_test.cpp")).read()
    edges_block = toy[toy.index("std::vector<std::vector<int>> edges"):toy.index("int num_vertices")]
    edges = [[int(a), int(b)] for a, b in re.findall(r"\{(\d+),\s*(\d+)\}", edges_block)]
    ints = lambda s: [int(x) for x in re.findall(r"-?\d+", s)]
    assignment = ints(re.search(r"assignment = \{([^}]*)\}", toy).group(1))
    complex_assignment = ints(re.search(r"assignment = \{ (0, 0, 0, 1[^}]*)\}", toy).group(1))
    entropy = float(re.search(r"ENTROPY = ([0-9.]+)", toy).group(1))
    v1 = float(re.search(r"MDL_10_VERTICES_50_EDGES_V1 = ([0-9.]+)", ent).group(1))
    v2 = float(re.search(r"MDL_10_VERTICES_50_EDGES_V2 = ([0-9.]+)", ent).group(1))
    deg = dict(re.findall(r"EXPECT_EQ\(B\.(degrees(?:_out|_in)?\(\d\)), (\d+)\)", bmt))
    degrees = {k: int(v) for k, v in deg.items()}
    nbd = re.search(r"class ComplexExample.*?BlockDegreesAfterUpdates\.block_degrees_out = \{([^}]*)\};"
                    r".*?block_degrees_in = \{([^}]*)\};.*?block_degrees = \{([^}]*)\};", toy, re.S)
    delta7 = {f"{a},{b}": int(c) for a, b, c in
              re.findall(r"EXPECT_EQ\(delta\.get\((\d),(\d)\), (-?\d+)\)",
                         ftt[ftt.index("BlockmodelDeltasAreCorrect"):ftt.index("BlockmodelDeltasShouldSumUpToZero")])}
    delta6 = {f"{a},{b}": int(c) for a, b, c in
              re.findall(r"EXPECT_EQ\(delta\.get\((\d),(\d)\), (-?\d+)\)",
                         ftt[ftt.index("SpecialCaseBlockmodelDeltasAreCorrect"):])}
    merge_delta = {f"{a},{b}": int(c) for a, b, c in re.findall(r"EXPECT_EQ\(delta\.get\((\d),(\d)\), (-?\d+)\)", bmg)}
    fixture = {
        "source": "reference test/toy_example.hpp, test/entropy_test.cpp, test/blockmodel_test.cpp, "
                  "test/finetune_test.cpp, test/block_merge_test.cpp",
        "num_vertices": 11,
        "edges": edges,
        "assignment": assignment,
        "complex_assignment": complex_assignment,
        "mdl": entropy,
        "null_mdl_v1_E50": v1,
        "null_mdl_v2_V10_E50": v2,
        "degrees": degrees,
        "complex_move_6_to_0_degrees": {"out": ints(nbd.group(1)), "in": ints(nbd.group(2)),
                                         "total_compute_new_block_degrees": ints(nbd.group(3))},
        "delta_move_7_to_0_with_self_in": delta7,
        "delta_complex_move_6_from_3_to_0": delta6,
        "delta_merge_0_into_1": merge_delta,
    }
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "toy_example.json")
    with open(out, "w") as f:
        json.dump(fixture, f, indent=1)
    print(out)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SBP_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: make_toy_fixture.py <reference checkout> (or set SBP_REFERENCE_DIR)")
    main(ref)
