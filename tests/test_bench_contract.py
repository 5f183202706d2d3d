"""The JSON line of `bench.py --impl reference` (CPU only): one line with the
metric, unit and keys the benchmark contract names, the reference arm's
end-to-end block with no device copies, and silence on ranks other than 0."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ)
    env.update(env_extra)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--subjects",
                          "3000", "--steps", "2", "--warmup", "3"],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return [line for line in out.stdout.splitlines() if line.strip()]


def test_reference_line():
    lines = _run({})
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"].startswith("DB residues x queries / s")
    assert d["unit"] == "residues*queries/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["config"]["workload"] == "q500_vs_1M" and d["config"]["query_len"] == 500
    # the reference's own kernel host-compiled (oracle/_ref) where it was built, else the oracle port
    from oracle import refkernel
    assert d["cpu_baseline"]["kind"] == ("reference" if refkernel.available(2) else "port")
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # one query per step: the length-weighted rate is the value times the query length
    assert abs(d["residue_pairs_per_s"] - d["value"] * 500) <= 1e-6 * d["residue_pairs_per_s"]


def test_reference_other_ranks_stay_silent():
    assert _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []
