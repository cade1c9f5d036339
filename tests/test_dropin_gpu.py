"""The reference's own CLIs with the B200 backend linked in place of its
CUDA backends (snc_b200/adapter): snc_bench --compare-backends must report
the cuda-* rows as served by the GPU (no "(fallback)") with the cpu
backend's spike and event counts -- exactly for cuda-sort -- snc_train
--device cuda must train on the GPU, and snc_cotrain --device cuda must run
its e-prop rounds on the GPU and feed their activity statistics to the
reference's structural update (Connectome::structural_update).  Skipped where the binaries were not
built (they need the reference sources at build time)."""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu
BUILD = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "snc_b200",
                     "adapter", "_build")
BENCH = os.path.join(BUILD, "snc_bench")
BENCH_SIDE = os.path.join(BUILD, "snc_bench_side")
TRAIN = os.path.join(BUILD, "snc_train")
COTRAIN = os.path.join(BUILD, "snc_cotrain")


def compare(args, binary=BENCH):
    if not os.path.exists(binary):
        pytest.skip("reference CLIs not built")
    out = subprocess.run([binary] + args + ["--compare-backends"], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    rows = {}
    for line in out.stdout.splitlines():
        m = re.match(r"^(\S+)\s+(\d+)\s+(\d+)\s+([\d.]+)\s+([\d.]+)\s+(\S+)(.*)$", line)
        if m:
            rows.setdefault(m.group(1), []).append((int(m.group(2)), int(m.group(3)), m.group(6),
                                                    m.group(7).strip()))
    return rows, out.stdout


@pytest.mark.parametrize("args", [
    ["--structure", "static-snc", "--encoder", "poisson", "--num-steps", "50", "--num-samples", "64",
     "--hidden", "256"],
    ["--structure", "random-sparse", "--num-steps", "100", "--num-samples", "16", "--hidden", "512",
     "--synapse-budget", "200000", "--inhib", "0.5", "--decay", "0.95", "--delay", "3"],
    ["--structure", "dense", "--num-steps", "30", "--num-samples", "8", "--hidden", "128",
     "--refractory", "2"],
])
def test_snc_bench_compare_backends(args):
    rows, text = compare(args)
    cpu = rows["cpu"][0]
    for name in ("cuda-atomic", "cuda-bucket", "cuda-sort"):
        assert name in rows, text
        sp, ev, match, note = rows[name][0]
        assert "fallback" not in note, text
        assert match in ("exact", "approx"), text
    sp, ev, match, _ = rows["cuda-sort"][0]
    assert (sp, ev, match) == (cpu[0], cpu[1], "exact"), text


@pytest.mark.parametrize("args", [
    ["--structure", "static-snc", "--encoder", "poisson", "--num-steps", "50", "--num-samples", "64",
     "--hidden", "256"],
    ["--structure", "random-sparse", "--num-steps", "100", "--num-samples", "16", "--hidden", "512",
     "--synapse-budget", "200000", "--inhib", "0.5", "--decay", "0.95", "--delay", "3"],
])
def test_b200_backends_beside_the_reference_cuda_backend(args):
    """The reference's backend table extended with b200-* names (beside.py),
    its own cuda_backend.cu linked unchanged: one --compare-backends run has
    the reference's cuda-* rows computed by its own kernels and the b200-*
    rows by this backend, none falling back; b200-sort matches cpu exactly."""
    rows, text = compare(args, BENCH_SIDE)
    cpu = rows["cpu"][0]
    for name in ("openmp", "cuda-atomic", "cuda-bucket", "cuda-sort", "b200-atomic", "b200-bucket",
                 "b200-sort"):
        assert name in rows, text
        sp, ev, match, note = rows[name][0]
        assert "fallback" not in note, text
        assert match in ("exact", "approx"), text
    sp, ev, match, _ = rows["b200-sort"][0]
    assert (sp, ev, match) == (cpu[0], cpu[1], "exact"), text


def test_snc_train_device_cuda():
    if not os.path.exists(TRAIN):
        pytest.skip("reference CLIs not built")
    out = subprocess.run([TRAIN, "--dataset", "synthetic", "--device", "cuda", "--batch", "32",
                          "--lr", "1.0", "--epochs", "3", "--num-train", "512", "--num-test", "128",
                          "--hidden", "128"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    assert "device=cuda" in out.stdout and "fallback" not in out.stdout, out.stdout
    last = [l for l in out.stdout.splitlines() if re.match(r"^\s+3\s", l)]
    assert last, out.stdout
    test_acc = float(last[0].split()[3])
    assert test_acc > 0.3, out.stdout  # chance is 0.1


def test_snc_cotrain_device_cuda():
    """cotrain_main.cpp:226-246: each round trains on the GPU session, carries
    the weights back to the connectome and collects the per-synapse and
    per-neuron activity the prune / regrow step consumes."""
    if not os.path.exists(COTRAIN):
        pytest.skip("reference CLIs not built")
    out = subprocess.run([COTRAIN, "--device", "cuda", "--batch", "32", "--outer", "3", "--inner", "2",
                          "--grow", "60", "--num-train", "512", "--num-test", "128", "--hidden", "128",
                          "--structural-budget", "6000", "--lr", "1.0"],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    assert "device=cuda" in out.stdout and "fallback" not in out.stdout, out.stdout
    rounds = [l.split() for l in out.stdout.splitlines() if re.match(r"^\s+\d+\s+\d+\s+\d+\s+\d+\s", l)]
    assert len(rounds) == 3, out.stdout
    synapses = {int(r[1]) for r in rounds}
    assert len(synapses) == 1, out.stdout  # every pruned synapse regrown
    for r in rounds[:2]:
        assert int(r[2]) == 60 and int(r[3]) == 60, out.stdout
    assert int(rounds[-1][6]) > 0, out.stdout  # the GPU forward spiked
    assert float(rounds[-1][5]) > 0.2, out.stdout  # chance is 0.1
