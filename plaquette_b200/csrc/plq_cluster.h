// plq_cluster.h -- Swendsen-Wang / Wolff chains (plq_cluster.cu).
#pragma once
#include "plq_abi_internal.h"

int cluster_validate(const plq_chain_desc *d);
int cluster_create(plq_chain *c);
int cluster_sweep(plq_chain *c);
void cluster_free(plq_chain *c);
