// bq_elh.cu -- the edge-length-heuristic builder (gpuBuilder with
// BuildConfig::ELH, cuBQL/builder/cuda/elh_builder.h:22-556, dispatch
// cuBQL/builder/cuda/gpu_builder.h:54-59).
//
// The same binned builder as bq_sah.cu, compiled a second time with its
// heuristic switched: 8 bins per axis instead of 16, bins at
// (c - lo) / (hi - lo) (no 1e-20 term), and the cost measure of a box is the
// sum of its edge lengths instead of its surface area.  Everything else --
// the leaf-versus-split rule, the first strictly cheapest candidate, the
// stable partition, ascending primIDs in leaves -- is shared.
#define BQ_HEUR 1
#include "bq_sah.cu"
