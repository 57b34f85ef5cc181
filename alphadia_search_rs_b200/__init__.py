"""B200-native peak-group selection with the API of alphadia-search-rs.

    from alphadia_search_rs_b200 import (DIAData, SpecLibFlat, SelectionParameters,
                                         PeakGroupSelection, CandidateCollection)

The classes mirror the reference's pyo3 module for the selection path and for the two
stages that consume its candidates: scoring (ScoringParameters, PeakGroupScoring,
CandidateFeatureCollection) and quantification (QuantificationParameters,
PeakGroupQuantification, SpecLibFlatQuantified); the work runs in
``_lib/libads_gpu.so`` (CUDA, sm_100a) behind the C ABI of ``include/ads_gpu.h``.
"""
from .api import (CandidateCollection, CandidateFeatureCollection, DIAData, PeakGroupQuantification,
                  PeakGroupScoring, PeakGroupSelection, QuantificationParameters, ScoringParameters,
                  SelectionParameters, SpecLibFlat, SpecLibFlatQuantified, device_count,
                  gaussian_kernel, mz_grid)

__all__ = ["DIAData", "SpecLibFlat", "SelectionParameters", "PeakGroupSelection",
           "CandidateCollection", "ScoringParameters", "PeakGroupScoring",
           "CandidateFeatureCollection", "QuantificationParameters", "PeakGroupQuantification",
           "SpecLibFlatQuantified", "mz_grid", "gaussian_kernel", "device_count"]
__version__ = "0.1.0"
