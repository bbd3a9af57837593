"""Golden lambda schedules of QligFEP's get_lambdas (qligfep.py:414-445, with
sigmoid from functions.py:7), for the restatement in q_b200/lambda_placement.py.

qligfep.py cannot be imported without its workflow dependencies, so this
script takes the two functions' own source out of the reference files (ast)
and runs them unchanged; `self` is not used by get_lambdas.  Run here, where
the reference tree exists:

    python tests/golden/make_lambda_golden.py /path/to/reference
"""
import ast
import json
import os
import sys

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "qligfep_lambdas.json")


def _function(path, name, cls=None):
    tree = ast.parse(open(path).read())
    nodes = tree.body
    if cls:
        nodes = next(n for n in nodes if isinstance(n, ast.ClassDef) and n.name == cls).body
    fn = next(n for n in nodes if isinstance(n, ast.FunctionDef) and n.name == name)
    return ast.get_source_segment(open(path).read(), fn)


def main(ref: str):
    REF = os.path.join(ref, "src", "QligFEP")
    ns = {}
    exec(_function(os.path.join(REF, "functions.py"), "sigmoid"), ns)
    src = _function(os.path.join(REF, "qligfep.py"), "get_lambdas", cls="QligFEP")
    lines = src.split("\n")
    indent = len(lines[1]) - len(lines[1].lstrip())
    src = "\n".join([lines[0].strip()] + [l[indent - 4:] if l.strip() else l for l in lines[1:]])
    exec(src, ns)
    out = {s: {str(w): ns["get_lambdas"](None, w, s) for w in range(2, 41)}
           for s in ("sigmoidal", "linear", "exponential", "reverse_exponential")}
    json.dump(out, open(OUT, "w"), indent=0)
    print("wrote", OUT)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_lambda_golden.py /path/to/reference")
    main(sys.argv[1])
