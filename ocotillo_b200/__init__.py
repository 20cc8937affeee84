"""ocotillo_b200: B200-native engine for ocotillo's per-column, per-wavelength radiative
transfer (Saha ionization -> continuous H opacities -> Feautrier solve along z).

The compute path is the CUDA library liboco_b200.so behind the C ABI in include/oco.h;
this package is its Python binding (ctypes, with numpy host arrays or torch device
tensors).  There is no CPU fallback: if the library is missing, importing the binding
raises.
"""
from .engine import (Engine, Batch, Server, OcoError, FORM_PLAIN, FORM_STABLE, FORM_MIXED, LAYOUT_REFERENCE,
                     LAYOUT_LAMBDA_FASTEST, TILING_WARP_COLUMN, TILING_PACKED, calc_wavelength,
                     dense_batch_offsets, batch_offsets, load_library, format_e, deck_block_inputs, run_deck,
                     read_fortran_records, disk_inputs, disk_params)

__all__ = ["Engine", "Batch", "Server", "OcoError", "FORM_PLAIN", "FORM_STABLE", "FORM_MIXED", "LAYOUT_REFERENCE",
           "LAYOUT_LAMBDA_FASTEST", "TILING_WARP_COLUMN", "TILING_PACKED", "calc_wavelength",
           "dense_batch_offsets", "batch_offsets", "load_library", "format_e", "deck_block_inputs", "run_deck",
           "read_fortran_records", "disk_inputs", "disk_params"]
