"""Extract the reference's golden vectors for the PauliSum path into reference_tables.json.

Run in a checkout that has the reference mounted (``python tests/golden/make_golden.py
<path-to-ppvm>``).  It reads the reference's own Rust test files as text and records:

* the Clifford sign tables of ``PhasedPauliWord``
  (crates/ppvm-pauli-word/src/phase/clifford.rs, tests at lines 184-374),
* the word-level truth tables (crates/ppvm-pauli-word/src/word/clifford.rs:7-179),
* the same tables for lossy words, where a gate touching a lost qubit L leaves the word
  alone (crates/ppvm-pauli-word/src/loss/clifford.rs:10-207),
* the golden expectation values of crates/ppvm-pauli-sum/tests/trotter.rs:104 and
  tests/cnot.rs:27.

The committed JSON is what tests use; this script is not run by the tests.
"""

from __future__ import annotations

import json
import os
import re
import sys


def _tables(src: str, signed: bool, alphabet: str = "IXYZ") -> dict[str, list[list[str]]]:
    out: dict[str, list[list[str]]] = {}
    for m in re.finditer(r"fn test_(\w+)\(\)\s*\{(.*?)\n    \}", src, re.S):
        name, body = m.group(1), m.group(2)
        pat = rf'\("([+\-]?[{alphabet}]+)",\s*"([+\-]?[{alphabet}]+)"\)'
        pairs = re.findall(pat, body)
        if pairs:
            out[name] = [list(p) for p in pairs]
    return out


def main(root: str) -> None:
    phase = open(os.path.join(root, "crates/ppvm-pauli-word/src/phase/clifford.rs")).read()
    word = open(os.path.join(root, "crates/ppvm-pauli-word/src/word/clifford.rs")).read()
    loss = open(os.path.join(root, "crates/ppvm-pauli-word/src/loss/clifford.rs")).read()
    trotter = open(os.path.join(root, "crates/ppvm-pauli-sum/tests/trotter.rs")).read()
    cnot = open(os.path.join(root, "crates/ppvm-pauli-sum/tests/cnot.rs")).read()
    golden_trotter = float(re.search(r"const GOLDEN: f64 = ([0-9.eE+-]+);", trotter).group(1))
    golden_cnot = float(re.search(r"assert_relative_eq!\(state\.trace\(&pat\), ([0-9.eE+-]+)\)", cnot).group(1))
    data = {
        "source": "QuEraComputing/ppvm test files (read as text)",
        "phase_tables": _tables(phase.split("#[cfg(test)]", 1)[1], True),
        "word_tables": _tables(word.split("#[cfg(test)]", 1)[1], False),
        "loss_word_tables": _tables(loss.split("#[cfg(test)]", 1)[1], False, "IXYZL"),
        "golden_trotter_n4": golden_trotter,
        "golden_cnot": golden_cnot,
    }
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "reference_tables.json"), "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    print("wrote", {k: (len(v) if isinstance(v, dict) else v) for k, v in data.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the ppvm checkout>")
    main(sys.argv[1])
