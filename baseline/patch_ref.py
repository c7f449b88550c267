"""Copies the reference's sources into baseline/_ref/src (git-ignored; never
committed) and applies the measurement patches of its CUDA build:

  * a cudaEvent pair around RunGPUi's relaunch loop of OCTMPSKernel
    (src/main.cu:572-623), printed as "[GPU n] kernel loop: <ms> ms, <k>
    launches": the device time of the photon work, without the per-A-scan
    allocations, uploads and the host's 1-s polling (src/main.cu:740-744);
  * a cap of MAX_LAUNCHES relaunches per A-scan, so that a packet that never
    ends (the reference has no step limit) cannot keep the loop going.

The kernel's source, its arithmetic and every other line are unchanged.

    python baseline/patch_ref.py <reference tree> <out dir>
"""
import os
import shutil
import sys

MAX_LAUNCHES = 20000

LOOP = "    for (int i = 1; *HostMem->n_photons_left > 0; ++i) {\n"
LAUNCH = "        OCTMPSKernel << < dimGrid, dimBlock >> > (DeviceMem, tstates);\n"
DONE = '    printf("[GPU %u] simulation done!\\n", hstate->dev_id);\n'


def patch_main(src):
    for anchor in (LOOP, LAUNCH, DONE):
        if src.count(anchor) != 1:
            raise SystemExit(f"patch anchor not found exactly once: {anchor!r}")
    src = src.replace(LOOP, (
        "    cudaEvent_t octmps_ev0, octmps_ev1;\n"
        "    cudaEventCreate(&octmps_ev0);\n"
        "    cudaEventCreate(&octmps_ev1);\n"
        "    int octmps_launches = 0;\n"
        "    cudaEventRecord(octmps_ev0);\n"
        + LOOP +
        f"        if (octmps_launches >= {MAX_LAUNCHES}) {{\n"
        "            fprintf(stderr, \"[GPU %u] relaunch cap reached\\n\", hstate->dev_id);\n"
        "            exit(2);\n"
        "        }\n"))
    src = src.replace(LAUNCH, LAUNCH + "        ++octmps_launches;\n")
    src = src.replace(DONE, (
        "    cudaEventRecord(octmps_ev1);\n"
        "    cudaEventSynchronize(octmps_ev1);\n"
        "    float octmps_ms = 0.0f;\n"
        "    cudaEventElapsedTime(&octmps_ms, octmps_ev0, octmps_ev1);\n"
        "    printf(\"[GPU %u] kernel loop: %f ms, %d launches\\n\", hstate->dev_id, octmps_ms,\n"
        "           octmps_launches);\n"
        + DONE))
    return src


def main():
    tree, out = sys.argv[1], sys.argv[2]
    os.makedirs(out, exist_ok=True)
    for fn in ("main.cu", "octmps_kernel.cuh", "octmps_kernel.h", "octmps.h", "bias.cpp",
               "octmps_io.cpp", "multithreading.h"):
        shutil.copyfile(os.path.join(tree, "src", fn), os.path.join(out, fn))
    p = os.path.join(out, "main.cu")
    with open(p) as f:
        src = f.read()
    with open(p, "w") as f:
        f.write(patch_main(src))


if __name__ == "__main__":
    main()
