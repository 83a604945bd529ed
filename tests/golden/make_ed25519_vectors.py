"""Regenerate tests/golden/ed25519_vectors.json from the reference's own Ed25519 tests.

The reference's known answers for its native verifier are the RFC 8032 section
7.1 TEST 1-3 vectors in crates/deep_ali/src/ed25519_verify.rs (tests
rfc8032_test1_empty_message .. rfc8032_test3_two_byte_message): public key,
signature and message as hex literals, and TEST 1's secret key in a comment.
This script reads them out of that file as text (nothing is run) so the tests
can pin the oracle's signer and verifier, and the library's verifier, to them.

Usage: python tests/golden/make_ed25519_vectors.py path/to/stark-stir-swarm
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _hexes(body):
    """hex("...") string literals of a test body, with Rust's line continuations joined"""
    return [re.sub(r"\\\s*\n\s*", "", m).replace("\n", "") for m in re.findall(r'hex(?:::<\d+>)?\(\s*"((?:[^"\\]|\\\s*\n)*)"', body)]


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_ed25519_vectors.py path/to/stark-stir-swarm")
    path = os.path.join(sys.argv[1], "crates", "deep_ali", "src", "ed25519_verify.rs")
    src = open(path).read()
    out = {"source": "stark-stir-swarm/crates/deep_ali/src/ed25519_verify.rs (RFC 8032 section 7.1 tests)",
           "vectors": []}
    for name in ("rfc8032_test1_empty_message", "rfc8032_test2_one_byte_message", "rfc8032_test3_two_byte_message"):
        start = src.index(f"fn {name}")
        body = src[start:src.index("#[test]", start) if "#[test]" in src[start:] else len(src)]
        hx = [h.replace(" ", "") for h in _hexes(body)]
        pub, sig = hx[0], hx[1]
        msg = hx[2] if len(hx) > 2 else ""
        v = {"test": name, "pub": pub, "sig": sig, "msg": msg}
        m = re.search(r"SECRET KEY:\s*([0-9a-f]{64})", body)
        if m:
            v["secret"] = m.group(1)
        assert len(pub) == 64 and len(sig) == 128, name
        out["vectors"].append(v)
    dst = os.path.join(HERE, "ed25519_vectors.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {dst}: {len(out['vectors'])} vectors")


if __name__ == "__main__":
    main()
