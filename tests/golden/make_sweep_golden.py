"""Golden member lists of the reference's sweep expansion.

Runs the reference's own create_constant_dictionnary and compute_value_len
(main_code/setup_simulation.py:17-47; only these two function definitions are
executed, not the script's folder-creating top level) on a few parameter
dictionaries and stores the expanded members, in order, as
tests/golden/sweep_expand.json.

    python tests/golden/make_sweep_golden.py
"""
import ast
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("PFAG_REFERENCE_DIR", "/root/reference")

CASES = [
    {"ncells": np.array([6]), "eta": np.array([0.03, 0.05]), "friction": np.array([1.0, 2.0, 4.0])},
    {"a": 1.0, "b": np.array([1.0, 2.0]), "c": np.array([3.0, 4.0]), "d": np.array([5.0])},
    {"x": np.array([1.0, 2.0, 3.0]), "y": np.array([7.0, 8.0, 9.0]), "z": np.array([0.5, 0.25])},
    {"p": np.array([1.0]), "q": np.array([2.0]), "r": np.array([3.0, 4.0, 5.0, 6.0])},
]


def main():
    src = open(os.path.join(REF, "main_code", "setup_simulation.py")).read()
    tree = ast.parse(src)
    funcs = [n for n in tree.body if isinstance(n, ast.FunctionDef)
             and n.name in ("compute_value_len", "create_constant_dictionnary")]
    ns = {"np": np}
    exec(compile(ast.Module(body=funcs, type_ignores=[]), "setup_simulation.py", "exec"), ns)
    out = []
    for case in CASES:
        members = ns["create_constant_dictionnary"](case)
        out.append({"input": {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in case.items()},
                    "members": [{k: float(v) for k, v in m.items()} for m in members]})
    with open(os.path.join(HERE, "sweep_expand.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(len(out), "cases")


if __name__ == "__main__":
    main()
