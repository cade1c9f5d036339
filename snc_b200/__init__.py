"""snc_b200 -- B200 (sm_100a) execution and training core for the SNC spiking
substrate (blazer502/snc), behind the reference's own interfaces.

Modules
  graph      host SNNGraph (CSR), SNCG wire format, InputEvent dtype
  runtime    snc::forward / Backend mirror, device graphs, batched runs,
             delivery autotuner
  eprop      cudatrain:: mirror (minibatch e-prop)
  bptt       surrogate-gradient BPTT (torch.autograd.Function + models)
  workloads  seeded synthetic graphs and inputs of the benchmark configs
"""
from .graph import EVENT_DTYPE, SNNGraph, load_graph, save_sncg, graph_from_sncg  # noqa: F401

__all__ = ["EVENT_DTYPE", "SNNGraph", "load_graph", "save_sncg", "graph_from_sncg"]
