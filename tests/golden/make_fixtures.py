"""Regenerate the golden fixtures in this directory from the reference checkout.

Writes:
  openhtj2k.json        the two OpenHTJ2K conformance codestreams the reference
                        pins its HT decoder with, plus their expected 8-bit
                        samples (crates/signinum-j2k-native/fixtures/htj2k/,
                        used by crates/signinum-j2k-native/src/lib.rs:2933-2947);
  ht_lookup_sha256.json SHA-256 of the reference's four packed HT lookup tables
                        (crates/signinum-j2k-native/src/j2c/ht_tables.rs:3,92,181,211),
                        each hashed as little-endian u16, so tests can check that
                        the tables this library builds are the same bits;
  ebcot_tables_sha256.json  SHA-256 of the reference's classic Tier-1 tables:
                        the three zero-coding context tables and the sign-coding
                        (label, xor) table (crates/signinum-j2k-native/src/j2c/
                        bitplane.rs:1152-1238) as u8 arrays, and the MQ
                        probability table (arithmetic_decoder.rs:333-386) as
                        little-endian (u16 qe, u8 nmps, u8 nlps, u8 switch)
                        records;
  LICENSE.OpenHTJ2K     the licence that travels with the conformance data.

Run only where the reference checkout exists:
    python tests/golden/make_fixtures.py <frames-sg/signinum checkout>
"""
import hashlib
import json
import pathlib
import re
import shutil
import struct
import sys


def main():
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <frames-sg/signinum checkout>")
    ref = pathlib.Path(sys.argv[1])
    here = pathlib.Path(__file__).parent
    fx = ref / "crates/signinum-j2k-native/fixtures/htj2k"
    out = {
        "source": "OpenHTJ2K conformance data (ds0_ht_*_b11), as checked into "
                  "frames-sg/signinum crates/signinum-j2k-native/fixtures/htj2k; "
                  "expected samples decoded with OpenJPH (see that directory's README).",
        "fixtures": {},
    }
    for name in ("openhtj2k_ds0_ht_12_b11", "openhtj2k_ds0_ht_09_b11"):
        out["fixtures"][name] = {
            "j2k_hex": (fx / (name + ".j2k")).read_bytes().hex(),
            "gray_hex": (fx / (name + ".gray")).read_bytes().hex(),
        }
    (here / "openhtj2k.json").write_text(json.dumps(out, indent=1) + "\n")
    shutil.copyfile(fx / "LICENSE.OpenHTJ2K", here / "LICENSE.OpenHTJ2K")

    text = (ref / "crates/signinum-j2k-native/src/j2c/ht_tables.rs").read_text()
    hashes = {}
    for name in ("VLC_TABLE0", "VLC_TABLE1", "UVLC_TABLE0", "UVLC_TABLE1"):
        m = re.search(r"const %s: \[u16; (\d+)\] = \[(.*?)\];" % name, text, re.S)
        vals = [int(v, 16) for v in re.findall(r"0x[0-9A-Fa-f]+", m.group(2))]
        blob = struct.pack("<%dH" % len(vals), *vals)
        hashes[name] = {"len": len(vals), "sha256": hashlib.sha256(blob).hexdigest()}
    (here / "ht_lookup_sha256.json").write_text(json.dumps(hashes, indent=1) + "\n")

    text = (ref / "crates/signinum-j2k-native/src/j2c/bitplane.rs").read_text()
    ebcot = {}
    for name in ("ZERO_CTX_LL_LH_LOOKUP", "ZERO_CTX_HL_LOOKUP", "ZERO_CTX_HH_LOOKUP"):
        m = re.search(r"const %s: \[u8; 256\] = \[(.*?)\];" % name, text, re.S)
        vals = [int(v) for v in re.findall(r"\d+", m.group(1))]
        ebcot[name] = {"len": len(vals), "sha256": hashlib.sha256(bytes(vals)).hexdigest()}
    m = re.search(r"const SIGN_CONTEXT_LOOKUP: \[\(u8, u8\); 256\] = \[(.*?)\];", text, re.S)
    pairs = [(int(a), int(b)) for a, b in re.findall(r"\((\d+),\s*(\d+)\)", m.group(1))]
    ebcot["SIGN_CONTEXT_LOOKUP"] = {
        "len": len(pairs),
        "label_sha256": hashlib.sha256(bytes(a for a, _ in pairs)).hexdigest(),
        "xor_sha256": hashlib.sha256(bytes(b for _, b in pairs)).hexdigest()}
    text = (ref / "crates/signinum-j2k-native/src/j2c/arithmetic_decoder.rs").read_text()
    m = re.search(r"static QE_TABLE: \[QeData; 47\] = qe!\((.*?)\);", text, re.S)
    rows = re.findall(r"(0x[0-9A-Fa-f]+),\s*(\d+),\s*(\d+),\s*(true|false)", m.group(1))
    blob = b"".join(struct.pack("<HBBB", int(q, 16), int(a), int(b), sw == "true") for q, a, b, sw in rows)
    ebcot["QE_TABLE"] = {"len": len(rows), "sha256": hashlib.sha256(blob).hexdigest()}
    (here / "ebcot_tables_sha256.json").write_text(json.dumps(ebcot, indent=1) + "\n")
    print("fixtures written to", here)


if __name__ == "__main__":
    main()
