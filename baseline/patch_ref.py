"""Copies the reference's sources into baseline/_ref/src (git-ignored; never
committed) and applies the measurement patches of its CUDA build:

  * a cudaEvent pair around RunGPUi's relaunch loop of OCTMPSKernel
    (src/main.cu:572-623), printed as "[GPU n] kernel loop: <ms> ms, <k>
    launches": the device time of the photon work, without the per-A-scan
    allocations, uploads and the host's 1-s polling (src/main.cu:740-744);
  * a cap of MAX_LAUNCHES relaunches per A-scan, so that a packet that never
    ends (the reference has no step limit) cannot keep the loop going.

  * the reference selects its launch settings for "compute capability 3.5"
    (600 threads per block) by defining the compiler's own __CUDA_ARCH__
    macro to 350 in src/octmps_kernel.h:61 and testing it in :67-97 and
    src/main.cu:978; defined in the host pass that macro marks host code
    as device code to CUDA's headers and to the launch stubs nvcc appends, and
    the build crashes at run time.  The same selection is made through a macro
    of its own (OCTMPS_REF_ARCH 350): same 600-thread blocks, same settings.

  * RunGPUi fills the device arrays rootIdx and rootIdx_cont (n_threads
    words each) by copying n_threads words from the address of the single
    host word hstate->rootIdx (src/main.cu:309, 327): a read far past the
    end of a small heap block, which faults on this host.  The copies come
    from a host buffer holding the root index n_threads times (what the code
    evidently means; InitThreadState overwrites both arrays per thread
    anyway, src/octmps_kernel.cuh:1119-1122).

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


ROOT_COPY = "    checkCudaErrors(cudaMemcpy(d_rootIdx, h_rootIdx, size,\n"
ROOT_COPY_CONT = "    checkCudaErrors(cudaMemcpy(d_rootIdx_cont, h_rootIdx, size,\n"
PHOTON_SECTION = "    // photon structure\n"


def patch_root_copies(src):
    for anchor in (ROOT_COPY, ROOT_COPY_CONT, PHOTON_SECTION):
        if src.count(anchor) != 1:
            raise SystemExit(f"patch anchor not found exactly once: {anchor!r}")
    src = src.replace(ROOT_COPY, (
        "    UINT32 *octmps_roots = (UINT32 *) malloc(size);\n"
        "    for (UINT32 octmps_i = 0; octmps_i < n_threads; ++octmps_i)\n"
        "        octmps_roots[octmps_i] = *h_rootIdx;\n"
        "    checkCudaErrors(cudaMemcpy(d_rootIdx, octmps_roots, size,\n"))
    src = src.replace(ROOT_COPY_CONT,
                      "    checkCudaErrors(cudaMemcpy(d_rootIdx_cont, octmps_roots, size,\n")
    src = src.replace(PHOTON_SECTION, "    free(octmps_roots);\n" + PHOTON_SECTION)
    return src


def patch_main(src):
    src = patch_root_copies(src)
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


ARCH_DEFINE = "#define __CUDA_ARCH__ 350 //mrei\n"


def patch_kernel_h(src):
    if src.count(ARCH_DEFINE) != 1:
        raise SystemExit("patch anchor not found exactly once: the __CUDA_ARCH__ define")
    src = src.replace(ARCH_DEFINE, "#define OCTMPS_REF_ARCH 350\n")
    head, sep, rest = src.partition("#define OCTMPS_REF_ARCH 350\n")
    # the tests of the setting below the define (the _WIN32 branch is left alone)
    rest = rest.replace("#ifndef __CUDA_ARCH__", "#ifndef OCTMPS_REF_ARCH")
    rest = rest.replace("#if __CUDA_ARCH__ ==", "#if OCTMPS_REF_ARCH ==")
    rest = rest.replace("#elif __CUDA_ARCH__ ==", "#elif OCTMPS_REF_ARCH ==")
    rest = rest.replace("(__CUDA_ARCH__ ==", "(OCTMPS_REF_ARCH ==")
    return head + sep + rest


def main():
    tree, out = sys.argv[1], sys.argv[2]
    os.makedirs(out, exist_ok=True)
    for fn in ("main.cu", "octmps_kernel.cuh", "octmps_kernel.h", "octmps.h", "bias.cpp",
               "octmps_io.cpp", "multithreading.h"):
        shutil.copyfile(os.path.join(tree, "src", fn), os.path.join(out, fn))
    p = os.path.join(out, "main.cu")
    with open(p) as f:
        src = f.read()
    cc_test = "if (cc[i] >= __CUDA_ARCH__) {"
    if src.count(cc_test) != 1:
        raise SystemExit("patch anchor not found exactly once: the compute-capability test")
    src = src.replace(cc_test, "if (cc[i] >= OCTMPS_REF_ARCH) {")
    with open(p, "w") as f:
        f.write(patch_main(src))
    p = os.path.join(out, "octmps_kernel.h")
    with open(p) as f:
        src = f.read()
    with open(p, "w") as f:
        f.write(patch_kernel_h(src))


if __name__ == "__main__":
    main()
