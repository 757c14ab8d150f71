// apply!(::QCircuit, state) with gate fusion: placeholder that applies the
// gates one by one until the tile engine lands.
#include "engine.h"

namespace vqc {

int apply_circuit_fused(vqc_state h, const vqc_gate* gates, int ngates, const double* mats) {
  for (int i = 0; i < ngates; ++i) {
    int rc = apply_gate_raw(h, gates[i].nq, gates[i].pos, mats + gates[i].mat);
    if (rc) return rc;
  }
  return VQC_OK;
}

}  // namespace vqc
