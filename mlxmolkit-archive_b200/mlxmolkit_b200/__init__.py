"""B200-native batched MMFF94/94s conformer optimizer (sm_100a CUDA behind a C ABI).

Drop-in for mlxmolkit's MMFF optimization surface:

* ``mmff_minimize_nk``                     (mlxmolkit/mmff_minimize.py:231)
* ``mmff_optimize_metal_multi_mol``        (mlxmolkit/mmff_metal_optimizer.py:217)
* ``mmff_optimize_metal_fused_multi_mol``  (mlxmolkit/mmff_metal_optimizer.py:543)
* ``generate_conformers_nk(run_mmff=True)`` (mlxmolkit/conformer_pipeline_v2.py:357)

Submodules are imported lazily so that term extraction and the synthetic
workload generator stay usable on machines without a GPU.
"""
from __future__ import annotations

import importlib

__all__ = [
    "MMFFParams", "extract_mmff_params", "mmff_minimize_nk",
    "mmff_optimize_metal_multi_mol", "mmff_optimize_metal_fused_multi_mol",
    "MetalBatchResult", "MultiMolResult", "generate_conformers_nk",
    "PipelineResult", "ConformerResult",
]

_LAZY = {
    "MMFFParams": "mmff_params", "extract_mmff_params": "mmff_params",
    "mmff_minimize_nk": "mmff_minimize",
    "mmff_optimize_metal_multi_mol": "mmff_metal_optimizer",
    "mmff_optimize_metal_fused_multi_mol": "mmff_metal_optimizer",
    "MetalBatchResult": "mmff_metal_optimizer", "MultiMolResult": "mmff_metal_optimizer",
    "generate_conformers_nk": "conformer_pipeline_v2",
    "PipelineResult": "conformer_pipeline_v2", "ConformerResult": "conformer_pipeline_v2",
}


def __getattr__(name):
    mod = _LAZY.get(name)
    if mod is None:
        raise AttributeError(name)
    return getattr(importlib.import_module(f"{__name__}.{mod}"), name)
