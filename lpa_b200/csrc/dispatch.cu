// Learned dispatch: placeholder hooks (the cost model is filled in by the
// learner module).
#include "runtime.h"

struct Learner {};

void lpa_learner_free(lpa_handle *h) {
  delete h->learner;
  h->learner = nullptr;
}
void lpa_learner_reset(lpa_handle *h) { lpa_learner_free(h); }
void lpa_learner_before_iteration(lpa_handle *) {}
void lpa_learner_after_iteration(lpa_handle *) {}
void lpa_learner_stats(lpa_handle *, lpa_stats *) {}
