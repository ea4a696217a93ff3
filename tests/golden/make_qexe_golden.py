"""Makes reference_qexe.json: the reference's own compiled example programs
(qoa_binaries/*.qx, *.oexe) as hex, for the bytecode front-end's tests.

For each binary whose .qoa source sits in the reference's qoa_files/, this
also assembles that source with qoa_b200.qexe.assemble (non-strict, skipping
lines as `qoa compile` skips lines it cannot parse) and records whether the
payload is byte-identical to the reference's binary. Run here, where the
reference tree is readable:  python tests/golden/make_qexe_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
REF = "/root/reference"

from qoa_b200 import qexe  # noqa: E402

SOURCES = {"hello.qx": "hello_world.qoa", "teleport.qx": "teleport.qoa", "shor.qx": "shor.qoa",
           "fusion.qx": "fusion-sim.qoa", "aes.qx": "aes-decryption.qoa",
           "aes-decryption-16.qx": "aes-decryption-16.qoa", "aes-22.qx": "aes-decryption-22.qoa"}


def main():
    out = {}
    bdir = os.path.join(REF, "qoa_binaries")
    for name in sorted(os.listdir(bdir)):
        data = open(os.path.join(bdir, name), "rb").read()
        rec = {"hex": data.hex()}
        src = SOURCES.get(name)
        if src and os.path.exists(os.path.join(REF, "qoa_files", src)):
            payload, skipped = qexe.assemble(open(os.path.join(REF, "qoa_files", src)).read(), strict=False)
            rec["assembler_matches_reference"] = payload == data[9:]
            rec["assembler_skipped_lines"] = len(skipped)
        out[name] = rec
    with open(os.path.join(HERE, "reference_qexe.json"), "w") as f:
        json.dump(out, f, indent=1)
    for k, v in out.items():
        print(k, len(v["hex"]) // 2, v.get("assembler_matches_reference"), v.get("assembler_skipped_lines"))


if __name__ == "__main__":
    main()
