"""Python restatement of the host half of the reference's largeIndex.

TEST INFRASTRUCTURE ONLY (the checker for tagore_large_merge). Follows
ZJU-DAILY/Tagore src/large_index.cu literally:
  reorder            :9-83    greedy cluster order and buffer slots
  order_merge_main   :86-106  pairwise cluster overlaps
  order_merge_new    :286-522 in-memory merge of a point's two copies,
                              eviction to spill files, final index file
and pybind.cu:314-330 for reading the centres file and forming clusters.
Where the reference reads an unset variable (no cluster with positive
overlap in reorder) the smallest unchosen cluster and slot 0 are used.
"""
import struct

import numpy as np


def clusters_from_centers(centers_path, num, cluster_num):
    cc = np.fromfile(centers_path, dtype=np.uint32, count=2 * num).reshape(num, 2)
    first, second = cc[:, 0].tolist(), cc[:, 1].tolist()
    clusters = [[] for _ in range(cluster_num)]
    for i in range(num):
        clusters[first[i]].append(i)
        clusters[second[i]].append(i)
    return first, second, clusters


def reorder(first, second, C, bs):
    inter = [dict() for _ in range(C)]
    for a, b in zip(first, second):
        inter[a][b] = inter[a].get(b, 0) + 1
        inter[b][a] = inter[b].get(a, 0) + 1
    bs = min(bs, C)
    visited = [False] * C
    result, buffer, position = [0], [0], [0] * C
    visited[0] = True
    for i in range(1, bs):
        max_sum, max_id = 0, None
        for j in range(C):
            if visited[j]:
                continue
            t = sum(inter[j].get(r, 0) for r in result)
            if t > max_sum:
                max_sum, max_id = t, j
        if max_id is None:
            max_id = visited.index(False)
        result.append(max_id)
        buffer.append(max_id)
        position[max_id] = i
        visited[max_id] = True
    for _ in range(C - bs):
        max_sum, max_id, max_evict = 0, None, 0
        for j in range(C):
            if visited[j]:
                continue
            best, best_k = 0, None
            for k in range(bs):
                t = 0
                l = k + 1
                while l % bs != k:
                    t += inter[j].get(buffer[l % bs], 0)
                    l += 1
                if t > best:
                    best, best_k = t, k
            if best > max_sum:
                max_sum, max_id, max_evict = best, j, best_k
        if max_id is None:
            max_id, max_evict = visited.index(False), 0
        buffer[max_evict] = max_id
        result.append(max_id)
        visited[max_id] = True
        position[max_id] = max_evict
    return result, position, bs


def merge(local_rows, medoids, first, second, clusters, order, position, bs, K, max_degree,
          spill):
    """Returns (index bytes, spill files {cid: bytes})."""
    C, N = len(clusters), len(first)
    pool = {}  # slot -> rows (list of lists [deg, ids...])
    buffer = [None] * bs
    pointers, visited, cached = [0] * N, [False] * N, [False] * N
    files = {}

    def slot_rows(cid):
        return pool[position[cid]]

    def do_spill(cid):
        out = bytearray()
        for j, node in enumerate(clusters[cid]):
            r = slot_rows(cid)[j]
            out += struct.pack("<I", r[0]) + struct.pack(f"<{r[0]}I", *r[1:1 + r[0]])
            visited[node] = True
            pointers[node] = None
        files[cid] = bytes(out)

    def load(i):
        cid = order[i]
        pool[position[cid]] = [list(r) for r in np.asarray(local_rows[cid]).reshape(-1, K)]

    load(0)
    for j, node in enumerate(clusters[order[0]]):
        visited[node] = True
        pointers[node] = j
    buffer[0] = order[0]
    for i in range(1, C):
        load(i)
        cur = order[i]
        for j, node in enumerate(clusters[cur]):
            if not visited[node]:
                visited[node] = True
                pointers[node] = j
                continue
            if pointers[node] is None:
                continue
            ano = second[node] if first[node] == cur else first[node]
            old_r = slot_rows(ano)[pointers[node]]
            new_r = slot_rows(cur)[j]
            a, b = (old_r, new_r) if first[node] != cur else (new_r, old_r)
            nhood, seen = [], set()
            for v in a[1:1 + a[0]]:
                seen.add(v)
                nhood.append(v)
            for v in b[1:1 + b[0]]:
                if v not in seen:
                    seen.add(v)
                    nhood.append(v)
            deg = min(len(nhood), max_degree)
            old_r[1:1 + deg] = nhood[:deg]
            old_r[0] = deg
            new_r[0] = 0
            cached[node] = True
        buffer[position[cur]] = cur
        if i >= bs - 1 and i + 1 < C:
            evict = buffer[position[order[i + 1]]]
            if evict is not None:
                do_spill(evict)
    for s in range(bs):
        if buffer[s] is not None:
            do_spill(buffer[s])
    streams = {c: memoryview(files[c]) for c in files}
    offs = {c: 0 for c in files}

    def read_u32(c, n=1):
        o = offs[c]
        vals = struct.unpack_from(f"<{n}I", streams[c], o) if n else ()
        offs[c] = o + 4 * n
        return list(vals)

    body, size = bytearray(), 0
    for i in range(N):
        if cached[i]:
            cid = first[i]
            (d1,) = read_u32(cid)
            if d1 == 0:
                cid = second[i]
                (d1,) = read_u32(cid)
            else:
                read_u32(second[i])
            ids = read_u32(cid, d1)
            body += struct.pack("<I", d1) + struct.pack(f"<{d1}I", *ids)
            size += 4 * (1 + d1)
        else:
            (d1,) = read_u32(first[i])
            a = read_u32(first[i], d1)
            (d2,) = read_u32(second[i])
            b = read_u32(second[i], d2)
            nhood, seen = [], set()
            for v in a:
                seen.add(v)
                nhood.append(v)
            for v in b:
                if v not in seen:
                    seen.add(v)
                    nhood.append(v)
            deg = min(len(nhood), max_degree)
            body += struct.pack("<I", deg) + struct.pack(f"<{deg}I", *nhood[:deg])
            size += 4 * (1 + deg)
    size += 24
    head = struct.pack("<QIIQ", size, max_degree, medoids[order[C - 1]], 0)
    return head + bytes(body), files
