"""Generate tests/golden/reference_tables.json from the turbo-metrics sources.

Run in a container where the reference tree is mounted (default path below, or
pass it as the first argument).  The JSON holds the numeric tables the
reference's SSIMULACRA2 path is defined by, parsed from its own sources, so
that the oracle and the CUDA engine can be pinned against them on machines
where the reference is absent:

  srgb8_lut        crates/ssimulacra2-cuda-kernel/src/srgb.rs:23-51 (256 f32)
  cpu_srgb8_table  crates/ssimulacra2-cuda/examples/cpu.rs:20-277 (256 f32)
  weights          crates/ssimulacra2-cuda/src/lib.rs:1023-1153 (108 f64)
  blur_consts      crates/ssimulacra2-cuda/examples/cpu.rs:931-948 (f32)
  corpus_scores    crates/ssim2-gpu/PORT_STATUS.md:28-33 -- scores of the CPU
                   crate ssimulacra2 0.5.1 on crates/dssim-cuda/test_data
"""
import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_tables.json")


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def floats_between(text, start_pat, end_pat="];"):
    i = text.index(start_pat)
    j = text.index("[", text.index("=", i)) + 1
    k = text.index(end_pat, j)
    body = re.sub(r"//[^\n]*", "", text[j:k])
    return [float(v.replace("_", "")) for v in re.findall(r"-?[0-9][0-9_]*\.?[0-9_]*(?:e-?[0-9]+)?", body)]


def main():
    srgb = read("crates/ssimulacra2-cuda-kernel/src/srgb.rs")
    lut = floats_between(srgb, "SRGB8_TO_LINEARF32_LUT")
    cpu = read("crates/ssimulacra2-cuda/examples/cpu.rs")
    cpu_lut = floats_between(cpu, "FROM_SRGB8_TABLE")
    lib = read("crates/ssimulacra2-cuda/src/lib.rs")
    weights = floats_between(lib, "const WEIGHT: [f64; 108]")
    consts = {}
    m = cpu[cpu.index("mod consts"):]
    m = m[: m.index("}")]
    for name, val in re.findall(r"pub const (\w+): \w+ = ([-0-9.e_]+)_(?:f32|usize)", m):
        consts[name] = float(val.replace("_", ""))
    status = read("crates/ssim2-gpu/PORT_STATUS.md")
    corpus = {}
    for q, cpu_s in re.findall(r"^\|\s*(\d+)\s*\|\s*(-?[0-9.]+)\s*\|", status, re.M):
        corpus["q%s" % q] = float(cpu_s)
    assert len(lut) == 256 and len(cpu_lut) == 256 and len(weights) == 108, (len(lut), len(cpu_lut), len(weights))
    out = {
        "source": "imazen/turbo-metrics (parsed by tests/golden/make_golden.py)",
        "srgb8_lut": lut,
        "cpu_srgb8_table": cpu_lut,
        "weights": weights,
        "blur_consts": consts,
        "corpus_scores_cpu_crate": corpus,
        "corpus_decoder_note": "scores produced by the image 0.25 JPEG decoder; other decoders may differ by +-1 per sample",
    }
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT, len(lut), len(weights), consts.keys(), corpus)


if __name__ == "__main__":
    main()
