/*
 * bnc_device_modifier.h -- the device-side interface of user modifiers.
 *
 * The reference lets a plugin register a host function for a modifier type ID
 * 0-127 (register_modifier_current, modifier_interface.h:38; the plugin table
 * overrides the built-in model of that ID, kernel_dispatch.h:336-343) and runs
 * it on the CPU only.  Here a user modifier is CUDA C++ source registered with
 * biocore_gpu_register_device_modifier / bnc_register_device_modifier
 * (bnc_b200.h): the library compiles it with NVRTC for sm_100a and launches its
 * kernel on the modifier's items.  There is no CPU fallback.
 *
 * The source includes this header and defines
 *
 *     extern "C" __global__ void my_entry(BncDeviceModifierArgs a) {
 *         unsigned int q = a.begin + blockIdx.x * blockDim.x + threadIdx.x;
 *         if (q >= a.end) return;
 *         BncSegmentState* s = a.seg + a.item_seg[q];
 *         float I = a.density[q] * (-70.0f - s->V);      // pA, + depolarising
 *         s->itot += (double)I;                          // the tick's I_total
 *     }
 *
 * One launch covers the items of this type in one modifier phase.  A phase holds
 * at most one modifier of any segment, so a kernel may read and write its item's
 * segment freely; the segment's modifiers in earlier slots have already run and
 * later slots run in later phases, which is the reference's slot order
 * (simulation_host.cpp:234-303).  The kernel adds its current to `itot`, as the
 * reference adds the returned current to I_total, and may change the item's state
 * words and the segment's V, ions and ATP as a ModifierFunc may.  `area` is the
 * effective area the reference stores in state[7].  Sources are compiled with
 * --fmad=false; they cannot include the C or C++ standard headers.
 */
#ifndef BNC_DEVICE_MODIFIER_H
#define BNC_DEVICE_MODIFIER_H

/* Per-segment working state of step 1 (96 bytes). */
typedef struct
#ifdef __CUDACC__
__align__(16)
#endif
{
    float V;              /* membrane potential, mV */
    float in[7];          /* intracellular Na, K, Ca, Cl, Mg, A-, H (mM) */
    float out[7];         /* extracellular, same order */
    float atp;            /* ATP level */
    float area;           /* membrane area, um^2 (the reference's state[7]) */
    unsigned int reserved;
    double vol;           /* volume, um^3 */
    double itot;          /* I_total of step 1 so far, pA: add the modifier's current */
    double reserved2;
} BncSegmentState;

typedef struct {
    BncSegmentState* seg;            /* per device segment */
    const unsigned int* item_seg;    /* item -> device segment */
    const float* density;            /* per item */
    float* state;                    /* [7][n_items]: word k of item q at state[k * n_items + q] */
    const float* nt;                 /* [15][n_seg] neurotransmitter, mM (read only in step 1) */
    unsigned int n_items, n_seg;
    unsigned int begin, end;         /* the items of this launch */
    float dt;                        /* ms */
    unsigned int type;               /* modifier type ID */
} BncDeviceModifierArgs;

#endif /* BNC_DEVICE_MODIFIER_H */
