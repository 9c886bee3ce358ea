// Bounds checks of the debug build (make CHECKS=1 -> libvdock_checked.so).
//
// compute-sanitizer is not available where this library is tested, so the
// checked build instruments the device indexing that the host validation is
// meant to make safe: a failed check records its code in a per-file device
// word (first failure wins) and the index is clamped into range, so the
// access stays in bounds; the host reads and clears the word after the
// call (take_device_checks) and fails the call with VD_ERR_CUDA and the
// code.  In the normal build the macros compile to nothing.
#pragma once

#include "common.h"

namespace vd {

#ifdef VD_CHECKS
static __device__ unsigned int vd_check_word;  // one per translation unit
#define VD_DCHECK(cond, code)                                        \
    do {                                                             \
        if (!(cond)) atomicCAS(&::vd::vd_check_word, 0u, unsigned(code)); \
    } while (0)
// idx clamped into [lo, hi], recording `code` when it was outside
#define VD_DCLAMP(idx, lo, hi, code) ::vd::dclamp((idx), (lo), (hi), (code))
__device__ __forceinline__ int dclamp(int idx, int lo, int hi, unsigned code) {
    if (idx < lo || idx > hi) {
        atomicCAS(&vd_check_word, 0u, code);
        return idx < lo ? lo : hi;
    }
    return idx;
}
static inline vd_status take_device_checks(const char* where) {
    unsigned int w = 0;
    VD_CUDA(cudaMemcpyFromSymbol(&w, vd_check_word, sizeof(w)));
    if (w) {
        const unsigned int z = 0;
        VD_CUDA(cudaMemcpyToSymbol(vd_check_word, &z, sizeof(z)));
        set_error(std::string(where) + ": device bounds check " + std::to_string(w) + " failed");
        return VD_ERR_CUDA;
    }
    return VD_OK;
}
#else
#define VD_DCHECK(cond, code) ((void)0)
#define VD_DCLAMP(idx, lo, hi, code) (idx)
static inline vd_status take_device_checks(const char*) { return VD_OK; }
#endif

// check codes
enum : unsigned {
    kChkPairAtom = 1,      // intra-pair atom index >= heavy atoms
    kChkPairType = 2,      // type-pair index >= 153
    kChkTableBin = 3,      // pair-table bin outside [0, 2047]
    kChkParent = 4,        // body parent outside [0, body)
    kChkAtomBody = 5,      // atom's body >= bodies
    kChkMapIndex = 6,      // trilinear corner outside the map
    kChkMapMissing = 7,    // no map for an atom's type
    kChkSubtree = 8,       // subtree atom range outside [0, atoms]
    kChkItem = 9,          // work item / ligand index outside the batch
    kChkGridRows = 10,     // grid tile touches more cell rows than staged
    kChkGridType = 11,     // staged receptor type outside the table slice
    kChkClusterKept = 12,  // kept chain index outside the ligand's chains
    kChkCell = 13,         // receptor cell index outside the cell grid
};

}  // namespace vd
