// plq_cluster.cu -- Swendsen-Wang and Wolff (placeholder until the labelling
// kernels land).
#include "plq_cluster.h"

int cluster_validate(const plq_chain_desc *) { return PLQ_OK; }
int cluster_create(plq_chain *) { return plq_fail(PLQ_EUNSUPPORTED, "cluster chains are not built yet"); }
int cluster_sweep(plq_chain *) { return plq_fail(PLQ_EUNSUPPORTED, "cluster chains are not built yet"); }
void cluster_free(plq_chain *) {}
