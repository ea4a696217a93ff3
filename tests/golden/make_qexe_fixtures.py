"""Makes qexe_programs.json: .qexe programs for the bytecode front-end's tests,
assembled by this repository's own assembler (qoa_b200.qexe) from the example
sources the reference ships as text (qoa_files/*.qoa).

Nothing here reads a compiled program: the fixture holds only what
qexe.assemble + qexe.write_exe produce from the .qoa sources, non-strict (a
line the assembler cannot encode is skipped, as `qoa compile` skips lines it
cannot parse; the count is recorded).

Run with the path of a planetryan/qoa checkout:

    python tests/golden/make_qexe_fixtures.py <path-to-qoa-checkout>
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from qoa_b200 import qexe  # noqa: E402

# fixture name -> source file under qoa_files/
SOURCES = {"hello_world": "hello_world.qoa", "teleport": "teleport.qoa", "shor": "shor.qoa",
           "aes-decryption-16": "aes-decryption-16.qoa", "fusion-sim": "fusion-sim.qoa"}


def main(argv):
    if len(argv) != 2:
        raise SystemExit(__doc__)
    src_dir = os.path.join(argv[1], "qoa_files")
    out = {}
    for name, src in sorted(SOURCES.items()):
        text = open(os.path.join(src_dir, src)).read()
        payload, skipped = qexe.assemble(text, strict=False)
        exe = qexe.write_exe(payload)
        out[name] = {"source": "qoa_files/" + src, "hex": exe.hex(), "skipped_lines": len(skipped),
                     "source_lines": len(text.splitlines())}
    with open(os.path.join(HERE, "qexe_programs.json"), "w") as f:
        json.dump(out, f, indent=1)
    for k, v in out.items():
        print(k, len(v["hex"]) // 2, "bytes,", v["skipped_lines"], "skipped of", v["source_lines"], "lines")


if __name__ == "__main__":
    main(sys.argv)
