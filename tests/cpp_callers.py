"""Builds the C++ callers under tests/cpp and writes the reference's file
formats (COLA graph and query files, type-1 edge lists, the config file)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
CPP = ROOT / "tests" / "cpp"
CUDA = Path("/usr/local/cuda")


def build(name: str, out_dir: Path, cuda: bool = False) -> Path:
    exe = out_dir / name
    cmd = ["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", str(CPP / f"{name}.cpp"), "-o",
           str(exe), f"-L{ROOT / 'vine_b200'}", "-lvine", f"-Wl,-rpath,{ROOT / 'vine_b200'}"]
    if cuda:
        cmd[4:4] = [f"-I{CUDA / 'include'}"]
        cmd += [f"-L{CUDA / 'lib64'}", "-lcudart"]
    subprocess.run(cmd, check=True)
    return exe


def write_cola_graph(path: Path, row_ptr, col, length, delay) -> None:
    """"N" then one "u: v w c ... -1" line per vertex (integral weights)."""
    n = len(row_ptr) - 1
    lines = [str(n)]
    for u in range(n):
        a, b = int(row_ptr[u]), int(row_ptr[u + 1])
        parts = [f"{u}:"]
        for j in range(a, b):
            parts.append(f"{int(col[j])} {int(length[j])} {int(delay[j])}")
        parts.append("-1")
        lines.append(" ".join(parts))
    path.write_text("\n".join(lines) + "\n")


def write_cola_queries(path: Path, src, dst, budget) -> None:
    path.write_text("".join(f"{int(s)} {int(t)} 0 0 {int(b)}\n" for s, t, b in zip(src, dst, budget)))


def write_config(path: Path, graph_type: int, graph: Path, queries: Path, ntask: int) -> None:
    path.write_text(f"{graph_type}\n{graph}\n{queries}\n{ntask}\n")


def parse_results(text: str):
    """Lines "task found cost delay n v0 .. v(n-1)" after "solve rc"."""
    out = {}
    started = False
    for ln in text.splitlines():
        if ln.startswith("solve "):
            started = True
            out["rc"] = int(ln.split()[1])
            continue
        if started and ln.strip():
            f = ln.split()
            n = int(f[4])
            out[int(f[0])] = {"found": bool(int(f[1])), "cost": float(f[2]), "delay": float(f[3]),
                              "path": np.array([int(x) for x in f[5:5 + n]], np.int64)}
    return out
