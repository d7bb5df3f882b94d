// Event-counting build of the narrow-phase kernels.  The kernels of
// narrowphase.cu are compiled a second time with RP3DG_COUNT_EVENTS, which
// makes every pair count the steps its code path takes (NpEvent: face tests,
// Gauss-map tests, edge distances, clip vertices, GJK iterations, ...) and add
// them to per-batch counters.  The namespace is renamed so both builds live in
// one library; the product kernels are not touched.  The counts, times the
// static per-event op table, give the FP32 work of a batch for the roofline.
#define RP3DG_COUNT_EVENTS 1
#define rp3dg rp3dg_ev
#include "narrowphase.cu"
