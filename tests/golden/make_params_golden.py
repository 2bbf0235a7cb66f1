"""Regenerate tests/golden/params_files.json from the reference's own parsers.

    make -C oracle REF=/root/reference/ParGeMSLR && python tests/golden/make_params_golden.py

For each format (sequential, parallel, hypre) and seed, tests/params_fuzz.py
writes a random parameter file; the reference parser of that format
(oracle/_ref/params_ref_<format>) reads it into an array filled with -7.5,
and the fixture keeps the file's SHA-256, the parser's status and every
slot it changed (JSON floats round-trip exactly).  Also kept, as values only:
the reference's default array (PargemslrSetDefaultParameterArray) and the
arrays it builds from its own five driver parameter files on top of it.
"""
import hashlib
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.paths import REFERENCE_TESTS as REF_TESTS  # noqa: E402
from tests import params_fuzz as F  # noqa: E402

REF_FILES = [("sequential", "sequential/inputs"), ("sequential", "sequential/inputs_ilut"),
             ("parallel", "parallel/inputs"), ("parallel", "parallel/inputs_bj_ilu"), ("hypre", "hypre/inputs")]
SEEDS = range(50)
FILL = -7.5


def main():
    out = {"fill": FILL, "cases": [], "reference_inputs": {}}
    d = tempfile.mkdtemp(prefix="pgx_params_")
    for fmt in F.FORMATS:
        for seed in SEEDS:
            text = F.random_file(fmt, seed)
            path = os.path.join(d, f"{fmt}_{seed}")
            with open(path, "w") as f:
                f.write(text)
            rc, vals = F.run_reference(fmt, path, FILL)
            changed = [[i, float(v)] for i, v in enumerate(vals) if not (v == FILL)]
            out["cases"].append({"format": fmt, "seed": seed, "sha256": hashlib.sha256(text.encode()).hexdigest(),
                                 "status": rc, "changed": changed})
    rc, vals = F.run_reference("sequential", os.devnull)
    assert rc == 0
    out["reference_inputs"]["defaults"] = {"format": None, "values": [float(v) for v in vals]}
    for fmt, rel in REF_FILES:
        rc, vals = F.run_reference(fmt, os.path.join(REF_TESTS, rel))
        assert rc == 0, rel
        out["reference_inputs"][rel] = {"format": fmt, "values": [float(v) for v in vals]}
    with open(os.path.join(HERE, "params_files.json"), "w") as f:
        f.write('{"fill": %s,\n"cases": [\n' % json.dumps(FILL))
        f.write(",\n".join(json.dumps(c, separators=(",", ":")) for c in out["cases"]))
        f.write('],\n"reference_inputs": {\n')
        f.write(",\n".join(f"{json.dumps(k)}: {json.dumps(v, separators=(',', ':'))}"
                           for k, v in out["reference_inputs"].items()))
        f.write("}}\n")
    n_err = sum(c["status"] != 0 for c in out["cases"])
    print(f"{len(out['cases'])} files ({n_err} rejected by the reference parser)")


if __name__ == "__main__":
    main()
