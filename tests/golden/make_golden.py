"""Extract the reference's known-answer vectors for the LSM hot path into golden.json.

    python tests/golden/make_golden.py <path of the reference source tree>

Every value is read from the reference's own test sources, as text, at the cited
lines; nothing is computed here. The committed golden.json is what the test suite reads, so the
tests never need the reference tree at run time.

Sources:
  philox      crates/finoptions-sim/src/random/philox.rs:120-130      Random123 KATs
  zignor      crates/finoptions-sim/src/random/normal.rs:115-142      16 pinned normal bit patterns
  moments     crates/finoptions-runtime/src/lib.rs:500-538            exact moment-kernel values
  dividends   crates/finoptions-core/src/dividend.rs:97-120           policy boundary values
  mesh        crates/finoptions-lsm/src/batch/pricing.rs:1319-1336    exact union mesh
  lsm         tests/test_lsm.py:29-270                                end-to-end fixtures
  one_div     crates/finoptions-lsm/src/policy.rs:1617-1670           statistical pin
              docs/adr/0006-independent-policy-lsm.md:49-53           its published summary
"""

from __future__ import annotations

import json
import re
import sys
from pathlib import Path


def _read(root: Path, rel: str) -> str:
    return (root / rel).read_text()


def _hex_words(text: str) -> list[int]:
    return [int(word.replace("_", ""), 16) for word in re.findall(r"0x[0-9a-fA-F_]+", text)]


def philox(root: Path) -> list[dict]:
    src = _read(root, "crates/finoptions-sim/src/random/philox.rs")
    block = src[src.index("fn matches_random123_known_answer_vectors") :]
    block = block[: block.index("#[test]", 10)]
    calls = re.findall(r"philox4x32_10\((.*?)\),\s*\[(.*?)\]", block, re.S)
    cases = []
    for args, expected in calls:
        if "u32::MAX" in args:
            counter, key = [0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2
        else:
            counter, key = [0, 0, 0, 0], [0, 0]
        cases.append({"counter": counter, "key": key, "output": _hex_words(expected)})
    return cases


def zignor(root: Path) -> dict:
    src = _read(root, "crates/finoptions-sim/src/random/normal.rs")
    block = src[src.index("fn pins_the_standard_normal_transform_sequence") :]
    header = re.search(r"PhiloxPathStream::new\((0x[0-9a-f_]+),\s*(0x[0-9a-f_]+),\s*(\d+),\s*(\d+)\)", block)
    assert header is not None
    seed, domain, path, count = header.groups()
    values_block = block[block.index("assert_eq!(") : block.index("]\n        );")]
    bits = _hex_words(values_block)
    return {
        "seed": int(seed.replace("_", ""), 16),
        "domain": int(domain.replace("_", ""), 16),
        "path": int(path),
        "count": int(count),
        "bits": bits,
    }


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the reference source tree>")
    root = Path(sys.argv[1])
    out = Path(__file__).with_name("golden.json")
    golden = {
        "philox": philox(root),
        "zignor": zignor(root),
        # runtime/src/lib.rs:500-506 and :522-537
        "moments": {
            "predictors": [0.5, 1.5],
            "responses": [2.0, 3.0],
            "basis": [-1.0, 2.0],
            "expected": [5.0, 4.0, 6.5],
        },
        "recurrence_moments": {
            "predictors": [0.5, 1.5],
            "responses": [2.0, 3.0],
            "previous": [0.0, 1.0],
            "current": [1.0, 2.0],
            "alpha": 0.5,
            "beta": 0.25,
            "next": [0.0, 1.75],
            "expected": [3.0625, 5.25, 4.59375],
        },
        # dividend.rs:97-120: (policy, amount, spot_before, spot_after)
        "dividend_policy": [
            ["liquidator", 5.0, 5.0, 0.0],
            ["survivor", 5.0, 5.0, 5.0],
            ["liquidator", 5.0, 2.0, 0.0],
            ["survivor", 5.0, 2.0, 2.0],
            ["liquidator", 5.0, 8.0, 3.0],
            ["survivor", 5.0, 8.0, 3.0],
        ],
        # pricing.rs:1319-1329
        "union_mesh": [
            {"maturity": 1.0, "base_intervals": 4, "cash": [0.1, 0.5, 0.9],
             "times": [0.0, 0.1, 0.25, 0.5, 0.75, 0.9, 1.0]},
            {"maturity": 1.0, "base_intervals": 2, "cash_bits_below_half": 1,
             "times_note": "[0, nextafter(0.5, 0), 0.5, 1]"},
        ],
        # tests/test_lsm.py:237-270 (declared continuation fixture) and :107-131 (origin decision)
        "insufficient_support_fixture": {
            "schedule_times": [0.0, 0.5, 1.0],
            "dividend_nodes": [1], "dividend_amounts": [7.0],
            "exercise_nodes": [1], "expiry_node": 2,
            "log_discounts": [0.0, -0.03, -0.06],
            "volatility": 0.30, "initial_spot": 100.0, "strike": 100.0,
            "paths": 4,
            "training": [10000, 1], "evaluation": [20000, 2],
            "expected_in_the_money_paths": 3, "expected_required_paths": 5,
            "expected_exercise_counts": [0, 4],
        },
        "origin_decision_fixture": {
            "schedule_times": [0.0, 0.5, 1.0],
            "dividend_nodes": [1], "dividend_amounts": [200.0],
            "exercise_nodes": [0], "expiry_node": 2,
            "log_discounts": [0.0, 0.0, 0.0],
            "volatility": 0.30, "initial_spot": 200.0, "strike": 100.0,
            "paths": 1000,
            "training": [10000, 1], "evaluation": [20000, 2],
            "expected_price": 100.0,
            "expected_exercise_counts": [1000, 0],
        },
        # policy.rs:1617-1670 / docs/adr/0006-independent-policy-lsm.md:226-231
        "one_dividend_statistical_pin": {
            "reference_value": 11.656448947710173,
            "rate": 0.06, "volatility": 0.30, "dividend": 7.0, "dividend_time": 0.5,
            "spot": 100.0, "strike": 100.0, "steps": 32,
            "replications": 12, "paths": 65536,
            "training_seed_base": 10000, "evaluation_seed_base": 20000,
            # docs/adr/0006-independent-policy-lsm.md:49-53 (published 8-decimal summary)
            "published_mean": 11.64337996,
            "published_replication_sd": 0.07366459,
            "published_standard_error": 0.02126514,
            "student_t_99_df_11": 3.1058065155392804,
        },
    }
    out.write_text(json.dumps(golden, indent=1) + "\n")


if __name__ == "__main__":
    main()
