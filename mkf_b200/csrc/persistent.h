// Persistent batch plans: the kernels of every product of a batch plan run
// as one launch of a persistent executor.  The plan records each lane's
// launches (kernel, grid, arguments) instead of issuing them; the executor's
// CTAs take (launch, block range) items from a queue in device memory and run
// the launch's kernel body on them, waiting (bounded) until the launch before
// it in the same lane has finished every item.
#pragma once

#include "common.cuh"

namespace mkf {

// The kernel bodies the executor runs.  Each stand-alone kernel that has a
// body registers its host stub under one of these (register_body), so a
// recorded launch of it can be found again.
enum BodyKind : int {
    kBodyNone = 0,
    kBodyCopyRows, kBodyFill,
    kBodyFwdCol6, kBodyFwdCol7, kBodyFwdCol8, kBodyFwdRow7, kBodyFwdRow8,
    kBodyInvCol6, kBodyInvCol7, kBodyInvCol8, kBodyInvRow7, kBodyInvRow8,
    kBodyDigitsCol6, kBodyDigitsCol7, kBodyDigitsCol8, kBodyRowIp7, kBodyRowIp8,
    kBodyDigitsPrep, kBodyModup4, kBodyModup8, kBodyModupSum4, kBodyModupSum8,
    kBodyCombine, kBodyKaratsuba, kBodyRescaleSpread, kBodyRescaleCombine, kBodyReplicate,
    kBodyIp111, kBodyIp121, kBodyIp221, kBodyIp211, kBodyIp112, kBodyIp122, kBodyIp222, kBodyIp212,
    kBodyCount
};

// Executor geometry: 512-thread CTAs, two per SM.  A 256-thread body runs
// two virtual blocks per CTA.  Dynamic shared memory per CTA: the largest
// body's (the fused row pass, or two digit column blocks).
constexpr int kPersThreads = 512;
constexpr size_t kPersSmemBytes = 3 * 4096 * 8;
constexpr size_t kPersArgBytes = 2048; // largest argument record

// One recorded launch.
struct PNode {
    int kind;            // BodyKind
    int threads;         // 512, or 256 (two bodies per CTA)
    unsigned nvb;        // virtual blocks: gx * gy * gz
    unsigned gx, gy, gz; // the launch's grid
    unsigned vpi;        // virtual blocks per item and body slot
    unsigned items;      // queue items: ceil(nvb / vpi) (512), ceil(nvb / (2 vpi)) (256)
    int dep;             // the node this one waits for (-1: none)
    unsigned dep_items;  // how many items of dep must have finished
    unsigned args;       // byte offset of the argument record in the blob
    unsigned args_bytes; // its size, a multiple of 16
    unsigned smem_words; // shared memory words of one body (offset of the second)
};
struct PItem {
    unsigned node, vb0; // the node and its first virtual block; a 512-thread
                        // item runs vb0 .. vb0+vpi-1, the halves of a
                        // 256-thread item vb0+h, vb0+h+2, ... (h = 0, 1)
};
// Control words: [0] queue head, [1] error flag, [2] first node whose wait
// expired + 1, [3] unused, then one finished-item counter per node.
constexpr int kCtlHead = 0, kCtlError = 1, kCtlStalled = 2, kCtlDone0 = 4;
struct PExec {
    const PNode *nodes;
    const PItem *items;
    const unsigned char *blob;
    unsigned nitems;
    unsigned *ctl;
    unsigned long long wait_ns; // bound of one wait
};

// Arguments of the executor's own bodies: recorded copies and fills.
struct CopyRowsArgs {
    uint64_t *dst;
    long long dst_stride;
    const uint64_t *src;
    long long src_stride;
    long long words;
    int rows;
};
struct FillArgs {
    unsigned char *p;
    unsigned long long bytes;
    int value;
};

// Registry of the bodies (host).
struct BodyInfo {
    int kind = kBodyNone;
    int threads = 0; // 0: launched with 256 or 512 threads, run as launched
    size_t smem_words = 0;
};
void register_body(const void *kernel, int kind, int threads, size_t smem_words);
bool find_body(const void *kernel, BodyInfo *out);

// CTAs of one executor launch on `device` (its resident slots); sets the
// executor's launch attributes on first use.  0 if it cannot run there.
int persistent_blocks(int device);
// Launches the executor over `e` on `st`.  Returns the CTAs launched, 0 on
// a launch error.
int launch_persistent(const PExec &e, int device, cudaStream_t st);

} // namespace mkf
