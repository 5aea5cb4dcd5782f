"""Compound grouping: the unit the reference's engine evaluates its
no-cutoff "immediate neighbour" pairs over.

The reference's builder splits every molecule into atom groups of at most 32
atoms by walking its bond tree (GroupAtoms2, code/LIMA_TOOLS/src/CompoundBuilder.cpp:425-514),
merges consecutive bonded groups into compounds while they fit
(CreateCompounds, CompoundBuilder.cpp:517-565) and records which compounds are
bonded to which.  Molecules of three atoms or fewer become single-site
"tinymols" unless their residue is "lxx" (CompoundBuilder.cpp:309-314); they
belong to no compound.  Each compound also gets two key particles and radii
(CompoundFactory.cpp:30-190) that the compound neighbour-list rule uses.

Where the reference's order depends on hash-set iteration (the order of a
molecule's bonds, CompoundBuilder.cpp:443-456), bonds are taken in ascending
index order here; on the chains of this package's systems the grouping is the
same either way except at ties between equally long sub-chains.
"""
from __future__ import annotations

import numpy as np

MAX_COMPOUND_PARTICLES = 32    # Constants.h:91
MAX_BONDED_COMPOUNDS = 6       # Bodies.cuh:205


def _next_permutation(a: list) -> bool:
    """std::next_permutation: the next lexicographic order in place; False when
    `a` was the last one (it is then reset to the first)."""
    i = len(a) - 2
    while i >= 0 and a[i] >= a[i + 1]:
        i -= 1
    if i < 0:
        a.reverse()
        return False
    j = len(a) - 1
    while a[j] <= a[i]:
        j -= 1
    a[i], a[j] = a[j], a[i]
    a[i + 1:] = reversed(a[i + 1:])
    return True


def _reorder_subchains(ids, down, space):
    """ReorderSubchains (CompoundBuilder.cpp:394-418): of the orders reachable by
    next_permutation from `ids`, the first that fits the most atoms into
    `space` when sub-chains are taken greedily."""
    best = list(ids)
    best_n = 0
    cur = list(ids)
    while True:
        n = 0
        for c in cur:
            if n + down[c] <= space:
                n += down[c]
        if n > best_n:
            best_n, best = n, list(cur)
        if not _next_permutation(cur):
            break
    return best


def _group_molecule(atoms, nbrs):
    """GroupAtoms2 for one molecule: atom ids in molecule order, nbrs[a] the
    neighbours of a in bond order.  Returns the list of atom groups."""
    root = atoms[0]
    # BFS tree (MoleculeGraph::ConstructMoleculeTree, MoleculeGraph.cpp:94-117)
    children = {root: []}
    order = [root]
    seen = {root}
    k = 0
    while k < len(order):
        cur = order[k]
        k += 1
        for nb in nbrs.get(cur, ()):
            if nb not in seen:
                seen.add(nb)
                children[nb] = []
                children[cur].append(nb)
                order.append(nb)
    # sub-tree sizes (ComputeNumDownstreamNodes, MoleculeGraph.cpp:120-142)
    down = {}
    for a in reversed(order):
        down[a] = 1 + sum(down[c] for c in children[a])

    def all_below(a):   # MoleculeTree::GetAllChildIdsAndSelf: stack order
        out, st = [], [a]
        while st:
            x = st.pop()
            out.append(x)
            st.extend(children[x])
        return out

    groups = [[]]
    stack = [root]
    while stack:
        node = stack.pop()
        if MAX_COMPOUND_PARTICLES - len(groups[-1]) == 0:
            groups.append([])
        groups[-1].append(node)
        kids = list(children[node])
        if kids:
            # the longest child chain continues the walk (first of equal ones)
            li = max(range(len(kids)), key=lambda i: (down[kids[i]], -i))
            stack.append(kids[li])
            kids[li] = kids[-1]
            kids.pop()
            for c in _reorder_subchains(kids, down, MAX_COMPOUND_PARTICLES - len(groups[-1])):
                if down[c] > MAX_COMPOUND_PARTICLES - len(groups[-1]):
                    groups.append([])
                groups[-1].extend(all_below(c))
    return groups


def build_compounds(system, tinymol_max_atoms: int = 0):
    """Compound of every atom (-1: none) and the bonded compound pairs of a
    lima_b200.systems.System.  Molecules are the connected components of the
    bond graph, in order of their first atom; molecules with at most
    `tinymol_max_atoms` atoms are tinymols (0: every molecule is "lxx" and
    becomes compounds, as the reference needs for charged water)."""
    n = system.n
    bonds = np.asarray(system.bonds, dtype=np.int64).reshape(-1, 2)
    nbrs = {}
    for a, b in bonds:
        nbrs.setdefault(int(a), []).append(int(b))
        nbrs.setdefault(int(b), []).append(int(a))
    # molecules: connected components, atoms ascending
    parent = list(range(n))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a, b in bonds:
        ra, rb = find(int(a)), find(int(b))
        if ra != rb:
            parent[max(ra, rb)] = min(ra, rb)
    mols = {}
    for i in range(n):
        mols.setdefault(find(i), []).append(i)
    # atom groups over all molecules, in molecule order
    groups = []
    for root in sorted(mols):
        atoms = mols[root]
        if len(atoms) <= tinymol_max_atoms:
            continue
        groups.extend(_group_molecule(atoms, nbrs))
    # consecutive groups joined by a bond (GroupAtoms2's last loop)
    bond_set = {(min(int(a), int(b)), max(int(a), int(b))) for a, b in bonds}

    def are_bonded(g0, g1):
        s1 = set(g1)
        for a in g0:
            for b in nbrs.get(a, ()):
                if b in s1 and (min(a, b), max(a, b)) in bond_set:
                    return True
        return False

    linked = [False] + [are_bonded(groups[i - 1], groups[i]) for i in range(1, len(groups))]
    # CreateCompounds: merge a group into the previous compound when bonded to it and it fits
    compound = np.full(n, -1, np.int32)
    gid_to_cid = []
    sizes = []
    for gi, g in enumerate(groups):
        if gi == 0 or not linked[gi] or sizes[-1] + len(g) > MAX_COMPOUND_PARTICLES:
            sizes.append(0)
        cid = len(sizes) - 1
        gid_to_cid.append(cid)
        sizes[-1] += len(g)
        compound[g] = cid
    pairs = set()
    for gi in range(1, len(groups)):
        if linked[gi] and gid_to_cid[gi] != gid_to_cid[gi - 1]:
            pairs.add((gid_to_cid[gi - 1], gid_to_cid[gi]))
    bonded = np.array(sorted(pairs), np.int32).reshape(-1, 2)
    return compound, bonded


def _hyper_dist(a, b, L):
    """The reference's FP32 hyper-position distance (BoundaryCondition.cuh:56-65)."""
    a = np.asarray(a, np.float32)
    m = np.asarray(b, np.float32).copy()
    L = np.float32(L)
    half = L / np.float32(2)
    m = m + L * ((a - m) > half).astype(np.float32)
    m = m - L * ((a - m) < -half).astype(np.float32)
    d = a - m
    return np.sqrt((d * d).sum(-1, dtype=np.float32))


def interaction_boundaries(system, compound):
    """Two key particles per compound (k-means, CompoundFactory.cpp:30-98) and
    their radii x 1.1 (clusterRadii, CompoundFactory.cpp:101-135, and
    CalcCompoundMetaInfo :164-190).  Returns (key atom indices (nc,2), radii
    (nc,2)), distances in FP32 with the reference's cubic-box rule (box edge
    system.box[0]).

    The reference seeds the second centre with index n_particles (one past the
    compound's atoms, a zero-initialised slot); here the seed is the atom
    farthest from the first one, which leads to the same kind of split.  The
    neighbour rule's guarantee below does not depend on the choice of keys:
    every atom lies within its key's radius by construction."""
    L = float(system.box[0])
    nc = int(compound.max()) + 1 if len(compound) and compound.max() >= 0 else 0
    keys = np.zeros((nc, 2), np.int64)
    radii = np.zeros((nc, 2), np.float32)
    pos = np.asarray(system.pos, np.float32)
    members = [[] for _ in range(nc)]
    for i, c in enumerate(compound):
        if c >= 0:
            members[c].append(i)
    for c in range(nc):
        idx = np.asarray(members[c])
        p = pos[idx]
        d0 = _hyper_dist(p[0], p, L)
        cent = [0, int(np.argmax(d0))]
        for _ in range(50):
            dist = np.stack([_hyper_dist(p[cent[j]], p, L) for j in range(2)], 1)
            lab = np.argmin(dist, 1)
            new = []
            for j in range(2):
                sel = p[lab == j]
                if len(sel) == 0:
                    new.append(cent[j])
                    continue
                mean = sel.mean(0, dtype=np.float32)
                new.append(int(np.argmin(_hyper_dist(p, mean[None, :], L))))
            if new == cent:
                break
            cent = new
        dist = np.stack([_hyper_dist(p[cent[j]], p, L) for j in range(2)], 1)
        lab = np.argmin(dist, 1)
        for j in range(2):
            sel = dist[lab == j, j]
            radii[c, j] = (sel.max() if len(sel) else 0.0) * np.float32(1.1)
            keys[c, j] = idx[cent[j]]
    return keys, radii
