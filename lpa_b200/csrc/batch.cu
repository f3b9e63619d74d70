// Batched graphs (placeholder until the persistent batch kernel lands).
#include "runtime.h"

extern "C" {
lpa_status lpa_batch_create(const lpa_graph_desc *, size_t, const lpa_opts *, struct lpa_batch **out) {
  if (out) *out = nullptr;
  return LPA_ERR_INVALID_ARG;
}
lpa_status lpa_batch_run(struct lpa_batch *, int, int, uint32_t *) { return LPA_ERR_INVALID_ARG; }
lpa_status lpa_batch_get_labels(struct lpa_batch *, size_t, uint32_t *, size_t) { return LPA_ERR_INVALID_ARG; }
lpa_status lpa_batch_destroy(struct lpa_batch *) { return LPA_ERR_INVALID_ARG; }
}
