"""CPU-side checks of the boundary: the C-ABI library builds, loads and
exports every symbol include/racon_b200.h declares; the command line keeps
racon's argument checks (test/racon_test.cpp:55-86 death tests)."""
import os
import re
import subprocess

import pytest

from conftest import ROOT, lambda_path

HEADER = os.path.join(ROOT, "include", "racon_b200.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rb_[a-z_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(native_lib):
    syms = subprocess.run(["nm", "-D", "--defined-only", native_lib.LIB_PATH], stdout=subprocess.PIPE,
                          text=True, check=True).stdout
    exported = set(re.findall(r" T (rb_[a-z_]+)", syms))
    missing = [s for s in _declared() if s not in exported]
    assert not missing, missing
    lib = native_lib.load()
    for s in _declared():
        assert hasattr(lib, s)


def _cli(*args):
    from racon_b200 import CLI_PATH
    return subprocess.run([CLI_PATH] + list(args), stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)


def test_cli_window_length_error(native_lib):
    r = _cli("-w", "0", "a.fasta", "b.paf", "c.fasta")
    assert r.returncode == 1
    assert "[racon::createPolisher] error: invalid window length!" in r.stderr


def test_cli_sequences_extension_error(native_lib):
    r = _cli("x.txt", "b.paf", "c.fasta")
    assert r.returncode == 1
    assert ("[racon::createPolisher] error: file x.txt has unsupported format extension (valid extensions: "
            ".fasta, .fasta.gz, .fna, .fna.gz, .fa, .fa.gz, .fastq, .fastq.gz, .fq, .fq.gz)!") in r.stderr


def test_cli_overlaps_extension_error(native_lib):
    r = _cli(lambda_path("sample_reads.fastq.gz"), "b.txt", "c.fasta")
    assert r.returncode == 1
    assert ("[racon::createPolisher] error: file b.txt has unsupported format extension (valid extensions: "
            ".mhap, .mhap.gz, .paf, .paf.gz, .sam, .sam.gz)!") in r.stderr


def test_cli_target_extension_error(native_lib):
    r = _cli(lambda_path("sample_reads.fastq.gz"), lambda_path("sample_overlaps.paf.gz"), "c.txt")
    assert r.returncode == 1
    assert "[racon::createPolisher] error: file c.txt has unsupported format extension" in r.stderr


def test_cli_missing_inputs(native_lib):
    r = _cli("a.fasta")
    assert r.returncode == 1
    assert "[racon::] error: missing input file(s)!" in r.stderr


def test_no_silent_cpu_path_without_gpu(native_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(native_lib.RaconB200Error):
        native_lib.Context(0)


def test_tuning_table_clamps_and_keeps_devices_apart(native_lib):
    # the per-device launch choices are host state: no device is needed to
    # set and read them, values outside their ranges are clamped, and one
    # device's choices do not touch another's
    before = [native_lib.tuning_get(d) for d in (5, 6)]
    try:
        native_lib.tuning_set(5, consensus_ctas_per_sm=9, consensus_order=7, alignment_warps_per_sm=1000)
        t = native_lib.tuning_get(5)
        assert (t["consensus_ctas_per_sm"], t["consensus_order"], t["alignment_warps_per_sm"]) == (3, 1, 32)
        native_lib.tuning_set(5, consensus_ctas_per_sm=0, consensus_order=0, alignment_warps_per_sm=6)
        t = native_lib.tuning_get(5)
        assert (t["consensus_ctas_per_sm"], t["consensus_order"], t["alignment_warps_per_sm"]) == (1, 0, 4)
        assert native_lib.tuning_get(6) == before[1]
    finally:
        native_lib.tuning_set(5, **before[0])


def test_tuning_defaults(native_lib):
    t = native_lib.tuning_get(7)
    assert (t["consensus_ctas_per_sm"], t["consensus_order"], t["alignment_warps_per_sm"], t["tuned"]) == (3, 0, 16, 0)
