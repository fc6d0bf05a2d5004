"""Extract the reference's known-answer constants into tests/golden/kats.json.

The reference (roynalnaruto/via-rs) ships its cross-language KAT constants as
Rust source (`pub const NAME: [u64; K] = [...]`) and a few PRG/sampler vectors
inline in its unit tests. This script reads those files *as text* and writes
the constants to JSON, so the test suite needs no access to the reference at
run time. Run it from the repository root:

    python tests/golden/make_golden.py /path/to/via-rs

Sources (paths relative to the reference root):
  crates/via-primitives/tests/data/layer3_kats.rs   switching
  crates/via-primitives/tests/data/layer4_kats.rs   gates
  crates/via-primitives/tests/data/layer5_kats.rs   LWE->RLWE conversion
  crates/via-integration/tests/data/layer6_kats.rs  QueryComp / RespComp
  crates/via-primitives/src/sampling/prg.rs         SHAKE-256 stream vectors
  crates/via-primitives/src/sampling/ternary.rs     ternary sampler vectors
  crates/via-primitives/src/sampling/uniform.rs     uniform_zq vectors
"""
import json
import pathlib
import re
import sys

FILES = {
    "layer3": "crates/via-primitives/tests/data/layer3_kats.rs",
    "layer4": "crates/via-primitives/tests/data/layer4_kats.rs",
    "layer5": "crates/via-primitives/tests/data/layer5_kats.rs",
    "layer6": "crates/via-integration/tests/data/layer6_kats.rs",
    "prg": "crates/via-primitives/src/sampling/prg.rs",
    "ternary": "crates/via-primitives/src/sampling/ternary.rs",
    "uniform": "crates/via-primitives/src/sampling/uniform.rs",
}

CONST_RE = re.compile(
    r"const\s+([A-Z0-9_]+)\s*:\s*\[(u8|u64|i8|i64)\s*;\s*(\d+)\s*\]\s*=\s*\[(.*?)\];", re.S
)


def parse_int(tok: str) -> int:
    tok = tok.strip().replace("_", "")
    neg = tok.startswith("-")
    if neg:
        tok = tok[1:]
    v = int(tok, 16) if tok.lower().startswith("0x") else int(tok)
    return -v if neg else v


def extract(text: str) -> dict:
    out = {}
    for name, _ty, count, body in CONST_RE.findall(text):
        body = re.sub(r"//[^\n]*", "", body)
        vals = [parse_int(t) for t in body.split(",") if t.strip()]
        if len(vals) != int(count):
            raise SystemExit(f"{name}: expected {count} values, got {len(vals)}")
        out[name] = vals
    return out


def main() -> None:
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <path of the via-rs checkout>")
    ref = pathlib.Path(sys.argv[1])
    golden = {}
    for group, rel in FILES.items():
        golden[group] = extract((ref / rel).read_text())
    dst = pathlib.Path(__file__).with_name("kats.json")
    dst.write_text(json.dumps(golden, indent=1, sort_keys=True) + "\n")
    n = sum(len(v) for v in golden.values())
    print(f"wrote {n} constants to {dst}")


if __name__ == "__main__":
    main()
