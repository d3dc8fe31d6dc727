"""Execution logs in the reference's CSV schemas for the Python multi-process drivers (the C++
drivers use include/dgt_logging.hpp, which follows the same rules):

    create_log_csv / write_line_to_file   src/Utilities/Logging.cpp:3-36
    calculate_gflops                      src/Utilities/GeneralUtilities.cpp:8-11
    NCCL 2.5D Cannon file name, header    src/25DCannonNCCL.cpp:335-338
    NCCL 2.5D Cannon row                  src/25DCannonNCCL.cpp:384-385

The header is written unless the file's first line is exactly the header; a file that
starts with any other line gets the header appended after its last line, as the reference
does.  Rows use the reference's printf conversions (%lf prints six decimals).
"""
from __future__ import annotations

import os
import socket

CANNON_NCCL_HEADER = ("Algo,M,N,K,TotalNodes,TotalGPUs,dRow,dCol,StackSize,DecompositionTime,ExecutionTime,"
                      "GatherTime,GFlops,DataLocation")


def cannon_nccl_log_name(machine: str, impl: str = "dgt") -> str:
    """'DGEMM_execution_logs-PreDistributed_GEMM-<machine>-2.5DCANNON-<impl>-NCCL.csv' (the
    reference's impl is 'cuBLAS')."""
    return f"DGEMM_execution_logs-PreDistributed_GEMM-{machine}-2.5DCANNON-{impl}-NCCL.csv"


def machine_name() -> str:
    """DGT_MACHINE_NAME from the environment, else the host name."""
    return os.environ.get("DGT_MACHINE_NAME") or socket.gethostname() or "unknown"


def slurm_num_nodes() -> int:
    """SLURM_JOB_NUM_NODES, or 1 when it is unset (the reference reads it unchecked)."""
    return int(os.environ.get("SLURM_JOB_NUM_NODES", "1"))


def calculate_gflops(M: int, N: int, K: int, seconds: float) -> float:
    return (2 * M * N * K * 1e-9) / seconds


def create_log_csv(path: str, header: str):
    """Opens `path` for appending, placing the header by the reference's rule."""
    f = open(path, "a+")
    f.seek(0)
    first = f.readline()
    if first != header + "\n":
        f.seek(0, os.SEEK_END)
        f.write(header + "\n")
    return f


def write_line_to_file(f, line: str) -> None:
    f.write(line)
    f.flush()


def cannon_nccl_row(algo, M, N, K, nodes, gpus, dRow, dCol, stack, decomp, execution, gather, gflops,
                    location="devices") -> str:
    """One row, formatted as "%s,%lld,%lld,%lld,%d,%d,%d,%d,%d,%lf,%lf,%lf,%lf,%s\\n"."""
    return "%s,%d,%d,%d,%d,%d,%d,%d,%d,%f,%f,%f,%f,%s\n" % (algo, M, N, K, nodes, gpus, dRow, dCol, stack, decomp,
                                                          execution, gather, gflops, location)
