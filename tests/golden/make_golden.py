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

DSSIM (the sibling metric sharing the linear-RGB pyramid):

  dssim.blur_kernel    crates/dssim-cuda-kernel/src/blur.rs:13-17 (3x3 f32)
  dssim.lab            crates/dssim-cuda-kernel/src/lab.rs:15-34 (f32 constants)
  dssim.c1, c2         crates/dssim-cuda-kernel/src/ssim.rs:18-19
  dssim.scale_weights  crates/dssim-cuda/src/lib.rs:77
  dssim.published      crates/dssim-gpu/PORT_STATUS.md:26-30 -- dssim-core 3.4
                       (CPU) and dssim-gpu scores of the parity_lock.rs cases
"""
import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TURBO_METRICS_REF", "/root/reference")
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
    dssim = dssim_tables()
    assert len(lut) == 256 and len(cpu_lut) == 256 and len(weights) == 108, (len(lut), len(cpu_lut), len(weights))
    out = {
        "source": "imazen/turbo-metrics (parsed by tests/golden/make_golden.py)",
        "srgb8_lut": lut,
        "cpu_srgb8_table": cpu_lut,
        "weights": weights,
        "blur_consts": consts,
        "corpus_scores_cpu_crate": corpus,
        "corpus_decoder_note": "scores produced by the image 0.25 JPEG decoder; other decoders may differ by +-1 per sample",
        "dssim": dssim,
    }
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT, len(lut), len(weights), consts.keys(), corpus)


def dssim_tables():
    blur = read("crates/dssim-cuda-kernel/src/blur.rs")
    kern = floats_between(blur, "const KERNEL")
    lab = read("crates/dssim-cuda-kernel/src/lab.rs")
    labc = {}
    for name, val in re.findall(r"^const (\w+): f32 = ([-0-9.e_]+);", lab, re.M):
        labc[name] = float(val.replace("_", ""))
    ssim = read("crates/dssim-cuda-kernel/src/ssim.rs")
    c = dict(re.findall(r"^const (C[12]): f32 = ([0-9.e-]+);", ssim, re.M))
    lib = read("crates/dssim-cuda/src/lib.rs")
    sw = floats_between(lib, "const SCALE_WEIGHTS")
    status = read("crates/dssim-gpu/PORT_STATUS.md")
    pub = {}
    names = {"32×32 identical gradient": "identical_32", "64×64 black vs white": "black_white_64",
             "64×64 noisy gradient (±8)": "noisy_gradient_64", "`dssim-cuda` corpus q70.jpg vs source.png": "q70",
             "`dssim-cuda` corpus q90.jpg vs source.png": "q90"}
    for label, cpu_s, gpu_s in re.findall(r"^\|\s*([^|]+?)\s*\|\s*([0-9.]+)\s*\|\s*([0-9.]+)\s*\|", status, re.M):
        if label in names:
            pub[names[label]] = {"dssim_core_cpu": float(cpu_s), "dssim_gpu": float(gpu_s)}
    assert len(kern) == 9 and len(sw) == 5 and len(pub) == 5 and "M_B_Z" in labc, (kern, sw, pub, labc)
    return {"blur_kernel": kern, "lab": labc, "c1": float(c["C1"]), "c2": float(c["C2"]), "scale_weights": sw,
            "published": pub}


if __name__ == "__main__":
    main()
