// plq_cluster.h -- Swendsen-Wang / Wolff chains (plq_cluster.cu).
#pragma once
#include "plq_abi_internal.h"

int cluster_validate(const plq_chain_desc *d);
int cluster_create(plq_chain *c);
int cluster_sweep(plq_chain *c);
// `sweeps` cluster sweeps (Wolff: `sweeps` single-cluster updates in one launch).
int cluster_sweep_n(plq_chain *c, uint64_t sweeps);
void cluster_free(plq_chain *c);
int cluster_labels(plq_chain *c, int32_t *out);
int cluster_size_histogram(plq_chain *c, int64_t *hist, int32_t nbins);
