// soil_slots.cuh — device helpers for the persistent per-neighbor slots of a
// soil_dev_view (soil_sys_enable_slots), for force hooks written in CUDA.
//
// The reference prototype's NeighborSlots (crates/soil_gpu/src/
// neighbor_slots.rs:19-184) gives every atom MAX_CONTACTS slots of (partner,
// payload), double-buffered: a kernel reads the OLD slots and writes the NEW
// ones each step, contacts not re-written are dropped, new contacts start at
// zero.  It keys a slot by the partner's index, which is valid only while no
// atom moves.  Here a slot is keyed by the partner's TAG, so a contact keeps
// its state through rebuilds, spatial sorts (the library moves each atom's
// slots with it) and periodic images (a ghost carries its local's tag).
//
// Ownership: the slots of a pair belong to the row atom i of the CSR half
// list (always local).  After a rebuild the pair can sit in the other atom's
// row; soil_slot_find then finds the old state in the partner's slots and
// says so, so that the consumer can reverse what depends on orientation.
// The atom of an incoming pair reads the same old slot (it does not write),
// so both ends of a pair see one state.
//
// Usage in a hook kernel, per local row atom i:
//   uint32_t k = 0;
//   for each partner j in row i with a contact:
//       double old[W]; int side = soil_slot_find(v, i, j, old);
//       ... new state from old (negate orientation-dependent parts if side < 0)
//       if (k < v.slot_max) soil_slot_put(v, i, k++, v.tag[j], state);
//   soil_slot_clear_from(v, i, k);
#pragma once

#include <stdint.h>

#include "soil_cuda.h"

#define SOIL_SLOT_NONE 0xFFFFFFFFu

// The local atom that owns atom a's slots: a, or the local a ghost images.
__device__ __forceinline__ uint64_t soil_slot_owner(const soil_dev_view& v, uint64_t a) {
    return a < v.nlocal ? a : (uint64_t)v.ghost_root[a - v.nlocal];
}

// Index of owner's old slot keyed by `partner_tag`, or -1.
__device__ __forceinline__ int soil_slot_index(const soil_dev_view& v, uint64_t owner,
                                               uint32_t partner_tag) {
    const uint32_t* t = v.slot_old_tag + owner * v.slot_max;
    for (uint32_t k = 0; k < v.slot_max; ++k)
        if (t[k] == partner_tag) return (int)k;
    return -1;
}

// Old state of the contact between row atom i (local) and atom j (local or
// ghost): i's slot keyed by tag[j] (returns +1), else the slot of j's owner
// keyed by tag[i] (returns -1: the state was written with the ends swapped),
// else none (returns 0).  Copies slot_width values to out (zeros for none).
__device__ __forceinline__ int soil_slot_find(const soil_dev_view& v, uint64_t i, uint64_t j,
                                              double* out) {
    const uint32_t W = v.slot_width;
    int side = 1;
    uint64_t owner = i;
    int k = soil_slot_index(v, i, v.tag[j]);
    if (k < 0) {
        side = -1;
        owner = soil_slot_owner(v, j);
        k = soil_slot_index(v, owner, v.tag[i]);
    }
    if (k < 0) {
        for (uint32_t c = 0; c < W; ++c) out[c] = 0.0;
        return 0;
    }
    const double* p = v.slot_old_val + (owner * v.slot_max + (uint64_t)k) * W;
    for (uint32_t c = 0; c < W; ++c) out[c] = p[c];
    return side;
}

// Write new slot k (< slot_max) of local atom i.
__device__ __forceinline__ void soil_slot_put(const soil_dev_view& v, uint64_t i, uint32_t k,
                                              uint32_t partner_tag, const double* val) {
    const uint64_t e = i * v.slot_max + k;
    v.slot_new_tag[e] = partner_tag;
    for (uint32_t c = 0; c < v.slot_width; ++c) v.slot_new_val[e * v.slot_width + c] = val[c];
}

// Mark new slots k.. of local atom i empty (after writing its k contacts).
__device__ __forceinline__ void soil_slot_clear_from(const soil_dev_view& v, uint64_t i,
                                                     uint32_t k) {
    for (; k < v.slot_max; ++k) v.slot_new_tag[i * v.slot_max + k] = SOIL_SLOT_NONE;
}
