"""The node order of a device-resident wave (graphflow_b200/include/graphflow/wave_order.hpp) on
the CPU: a transform forwards every chunk to one node, which then runs later in the same wave
wherever no cycle of transforms alone forbids it. Checked on the photon graph, chains in both
index directions, cycles, and random graphs (every order a permutation; every transform edge not
on a transform-only cycle points forward)."""
import os
import random
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NO = 2**32 - 1


@pytest.fixture(scope="module")
def order_binary(tmp_path_factory):
    out = tmp_path_factory.mktemp("wave_order") / "wave_order"
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-I", os.path.join(ROOT, "graphflow_b200", "include", "graphflow"),
           os.path.join(ROOT, "tests", "cpp", "wave_order.cpp"), "-o", str(out)]
    subprocess.run(cmd, check=True)
    return str(out)


def orders(binary, graphs):
    text = "".join(f"{len(f)} {' '.join(str(int(x)) for x in f)} {' '.join(str(s) for s in succ)}\n"
                   for f, succ in graphs)
    r = subprocess.run([binary], input=text, capture_output=True, text=True, timeout=60, check=True)
    return [[int(x) for x in line.split()] for line in r.stdout.splitlines()]


def on_transform_cycle(forwards, succ):
    n = len(forwards)
    edge = [forwards[k] and succ[k] < n and succ[k] != k for k in range(n)]
    cyc = set()
    for k in range(n):
        seen, v = [], k
        while edge[v] and v not in seen:
            seen.append(v)
            v = succ[v]
        if edge[v] and v in seen:
            cyc.update(seen[seen.index(v):])
    return cyc


def test_photon_graph(order_binary):
    # generate(0) -> propose flight(1, transform) -> advance and route(2, partition) ->
    # scatter(3, transform) -> propose flight; terminal(4, sink)
    forwards = [0, 1, 0, 1, 0]
    succ = [1, 2, NO, 1, NO]
    (seq,) = orders(order_binary, [(forwards, succ)])
    assert seq == [0, 3, 1, 2, 4]  # scatter, flight and route in one wave


@pytest.mark.parametrize("n", [1, 2, 5])
def test_chains(order_binary, n):
    up = ([1] * (n - 1) + [0], [k + 1 for k in range(n - 1)] + [NO])    # k -> k + 1
    down = ([0] + [1] * (n - 1), [NO] + [k - 1 for k in range(1, n)])   # k -> k - 1
    a, b = orders(order_binary, [up, down])
    assert a == list(range(n))
    assert b == list(range(n - 1, -1, -1))


def test_transform_cycles_keep_index_order(order_binary):
    cyc = ([1, 1, 1], [1, 2, 0])
    self_loop = ([1, 0], [0, NO])
    into_cycle = ([1, 1, 1, 1], [2, 3, 3, 2])  # 0 -> 2 <-> 3 <- 1
    a, b, c = orders(order_binary, [cyc, self_loop, into_cycle])
    assert a == [0, 1, 2]
    assert b == [0, 1]
    assert c == [0, 1, 2, 3]


def test_random_graphs(order_binary):
    rng = random.Random(7)
    graphs = []
    for _ in range(400):
        n = rng.randint(1, 12)
        forwards = [rng.random() < 0.6 for _ in range(n)]
        succ = [rng.randrange(n) if rng.random() < 0.85 else NO for _ in range(n)]
        graphs.append((forwards, succ))
    for (forwards, succ), seq in zip(graphs, orders(order_binary, graphs)):
        n = len(forwards)
        assert sorted(seq) == list(range(n))
        pos = {v: i for i, v in enumerate(seq)}
        cyc = on_transform_cycle(forwards, succ)
        for k in range(n):
            if forwards[k] and succ[k] < n and succ[k] != k and k not in cyc:
                assert pos[succ[k]] > pos[k], (forwards, succ, seq)
