"""Generates the golden fixtures: runs the reference's own search (compiled
from its unmodified sources by oracle/Makefile, FP64 and FP32 builds) on every
case of cases.py and stores its trigger records.

    python tests/golden/make_golden.py          (needs the reference tree; CPU only)

Each fixture <name>.npz holds: input checksum, the reference's records
(pm, m, n, s, ra, dec, fdot; lens; flat (f, F) pairs) for the f64 and f32
builds, and their walltimes.
"""
from __future__ import annotations

import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from tdfstat_b200 import synth  # noqa: E402
import refkit  # noqa: E402
from golden.cases import CASES, input_checksum  # noqa: E402


def pack(recs):
    lens = np.array([len(p) for p in recs.pairs], dtype=np.int64)
    flat = np.concatenate(recs.pairs).astype(np.float32) if len(recs.pairs) and lens.sum() else np.zeros(0, np.float32)
    return recs.hdr.astype(np.float32), lens, flat, recs.pm.astype(np.int32)


def main(names=None):
    refkit.build_oracle(ref=True)
    for name, case in CASES.items():
        if names and name not in names:
            continue
        root = tempfile.mkdtemp(prefix="tdfgold_")
        try:
            ini = synth.write_case(root, case)
            cks = input_checksum(root)
            out = {"checksum": np.array(cks)}
            for which in ("f64", "f32"):
                shutil.rmtree(os.path.join(root, "out"), ignore_errors=True)
                # write_case put the veto-line file in out/; regenerate it
                synth.write_case(root, case)
                recs, meta, _ = refkit.run_reference(ini, which, threads=1)
                hdr, lens, flat, pm = pack(recs)
                out[which + "_hdr"] = hdr
                out[which + "_lens"] = lens
                out[which + "_pairs"] = flat
                out[which + "_pm"] = pm
                out[which + "_walltime"] = np.array(meta.get("walltime", 0.0))
                print("%-20s %s: %d records, %d triggers, %.2fs" % (name, which, len(recs), recs.ntrig,
                                                                    meta.get("walltime", 0.0)))
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        finally:
            shutil.rmtree(root, ignore_errors=True)


def main_coinc(names=None):
    """Coincidence fixtures: the reference's search (FP64 build) on every
    segment, then its coincidence program (oracle/_ref/coinc-ref) on the
    segments' trigger files of one hemisphere, once per option set."""
    import subprocess
    from golden.cases import COINC_CASES, write_coinc_case
    refkit.build_oracle(ref=True)
    subprocess.run(["make", "-s", "-C", os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"), "coinc"],
                   check=True)
    for name, cc in COINC_CASES.items():
        if names and name not in names:
            continue
        root = tempfile.mkdtemp(prefix="tdfgoldc_")
        try:
            segs = write_coinc_case(root, name)
            out = {"checksum": np.array(input_checksum(root))}
            files = []
            for seg, ini in segs:
                refkit.run_reference(ini, "f64", threads=1)
                files.append("out/triggers_%03d_%04d_%d.h5" % (seg, cc["base"].band, cc["hemi"]))
            for key, o in cc["opts"].items():
                odir = os.path.join(root, "coin_" + key)
                os.makedirs(odir, exist_ok=True)
                ini = os.path.join(root, "coinc_%s.ini" % key)
                with open(ini, "w") as f:
                    f.write("[coincidences]\n")
                    for k, v in o.items():
                        f.write("%s = %r\n" % (k, v))
                    f.write("hemi = %d\nout_dir = %s\ntrig_file_list = %s\n" % (cc["hemi"], odir, " ".join(files)))
                subprocess.run([refkit.REF_BIN["coinc"], ini], cwd=root, check=True, capture_output=True)
                cf = [fn for fn in os.listdir(odir) if fn.startswith("coin_")]
                coin = refkit.read_coin_file(os.path.join(odir, cf[0]))
                for ish, blk in coin.items():
                    p = "%s_%02d_" % (key, ish)
                    cois = blk["coi"]
                    out[p + "seginfo"] = blk["seginfo"]
                    out[p + "w"] = np.array([c[0] for c in cois], dtype=np.int16)
                    out[p + "vals"] = np.array([c[1:6] for c in cois], dtype=np.float32).reshape(-1, 5)
                    out[p + "cseg"] = np.concatenate([c[6] for c in cois]) if cois else np.zeros(0, np.int16)
                    out[p + "trig"] = np.concatenate([c[7] for c in cois]) if cois else np.zeros(0, np.int32)
                    out[p + "ntrig"] = np.concatenate([c[8] for c in cois]) if cois else np.zeros(0, np.int16)
                print("%-10s %s: %s coincidences over 16 shifts" % (name, key, sum(len(b["coi"]) for b in coin.values())))
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        finally:
            shutil.rmtree(root, ignore_errors=True)


def main_vlines(names=None):
    """Veto-line fixtures: the veto file the reference's vlinegen program
    writes for each case of VLINE_CASES, as text (<name>.vlines)."""
    import subprocess
    from golden.cases import VLINE_CASES
    subprocess.run(["make", "-s", "-C", os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"), "vlinegen"],
                   check=True)
    for name, case in VLINE_CASES.items():
        if names and name not in names:
            continue
        root = tempfile.mkdtemp(prefix="tdfgoldv_")
        try:
            ini = synth.write_case(root, case)
            text = refkit.run_vlinegen(ini)
            with open(os.path.join(HERE, name + ".vlines"), "w", encoding="latin-1") as f:
                f.write("# input checksum %s\n" % input_checksum(root))
                f.write(text)
            print("%-12s %d veto lines" % (name, sum(1 for ln in text.splitlines() if not ln.startswith("#"))))
        finally:
            shutil.rmtree(root, ignore_errors=True)


if __name__ == "__main__":
    main(sys.argv[1:])
    main_coinc(sys.argv[1:])
    main_vlines(sys.argv[1:])
