"""Extracts the Liberty data of the synthetic workloads' cell mix from the
sky130hd typical-corner library into a compact JSON file shipped with the
package (the library itself is 12.8 MB and is not shipped).

Usage: python -m gtpower_b200.data.extract_cells <sky130hd_tt.lib>
"""
import os
import sys

from gtpower_b200 import liberty

SYNTH_CELLS = [
    "sky130_fd_sc_hd__inv_1",
    "sky130_fd_sc_hd__nand2_1",
    "sky130_fd_sc_hd__nor2_1",
    "sky130_fd_sc_hd__a21oi_1",
    "sky130_fd_sc_hd__xor2_1",
    "sky130_fd_sc_hd__mux2_1",
    "sky130_fd_sc_hd__dfxtp_1",
]

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sky130hd_tt_synth_cells.json")

if __name__ == "__main__":
    liberty.extract(sys.argv[1], SYNTH_CELLS, OUT)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")
