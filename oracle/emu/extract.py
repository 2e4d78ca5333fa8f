"""Copy the reference's CUDA kernel sources, unmodified, into oracle/_ref/.

TEST INFRASTRUCTURE ONLY (builds the checker that pins the oracle).

The reference keeps its TreePM kernels as one raw string,
CUDA_TWOPASS_KERNELS, in src/nbody_gpu_twopass.rs (lines 27-1813), compiled at
run time by NVRTC.  Its Poisson kernels live in cuda/cufft_wrapper.cu
(apply_green_kernel :148-208, normalize_kernel :290-295) next to cuFFT host
code.  This script writes the raw string to twopass_kernels.cu and the two
__global__ functions of cufft_wrapper.cu (brace-matched) to cufft_kernels.cu.
Nothing is edited: the harness compiles them with a CUDA emulation header.

usage: python extract.py <reference_root> <out_dir>
"""
import os
import sys


def extract_raw_string(path, name):
    text = open(path, encoding="utf-8").read()
    start_tok = "const %s: &str = r#\"" % name
    i = text.index(start_tok) + len(start_tok)
    j = text.index('\n"#;', i)
    return text[i:j + 1]


def extract_function(text, signature):
    i = text.index(signature)
    b = text.index("{", i)
    depth = 0
    for k in range(b, len(text)):
        if text[k] == "{":
            depth += 1
        elif text[k] == "}":
            depth -= 1
            if depth == 0:
                return text[i:k + 1] + "\n"
    raise ValueError("unbalanced braces after " + signature)


def main():
    ref, out = sys.argv[1], sys.argv[2]
    os.makedirs(out, exist_ok=True)
    tp = extract_raw_string(os.path.join(ref, "src", "nbody_gpu_twopass.rs"),
                            "CUDA_TWOPASS_KERNELS")
    with open(os.path.join(out, "twopass_kernels.cu"), "w") as f:
        f.write(tp)
    cw = open(os.path.join(ref, "cuda", "cufft_wrapper.cu"), encoding="utf-8").read()
    parts = [extract_function(cw, "__global__ void apply_green_kernel("),
             extract_function(cw, "__global__ void normalize_kernel(")]
    with open(os.path.join(out, "cufft_kernels.cu"), "w") as f:
        f.write("\n".join(parts))


if __name__ == "__main__":
    main()
