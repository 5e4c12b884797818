// Host side of the multifrontal factorization of a frame's implicit step (the kernels: bl_multifrontal.cuh).
//
// The reference factors the step's block system column by column, right-looking, with the exact minimum-degree order
// of its symbolic phase (frame_fem.cpp:2887-2920). The same order is kept here - the fill, and so the factor's
// nonzeros, are the reference's - but the columns are grouped into fronts: dense blocks factored with dense kernels,
// which is where a GPU is fast.
//  * Elimination tree: column k's parent is its first off-diagonal row.
//  * Fundamental supernodes: a column joins its parent's group when it is that parent's only child and its rows are the
//    parent and the parent's rows (the columns then share one dense structure).
//  * Relaxed amalgamation: a group merges into its parent group while the merged group stays small or adds few
//    explicit zeros (the thresholds below, in frame nodes: 6 degrees of freedom each).
//  * Each front holds its pivots (its columns) and its rows (the structure above them), both in elimination order, as
//    one dense lower triangle in degrees of freedom, column-major. Its factorization eliminates the pivots and leaves
//    the Schur complement of its rows in place, which its parent adds into its own front (extend-add).
//  * Fronts run level by level of the front tree (leaves first), every front of a level at once.
// The solution equals the column-by-column one up to the order of the floating-point sums.
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

namespace blg {

struct MfPlan {
    // per front, in execution order (by level, leaves first)
    std::vector<int> npiv, nrow;    // frame nodes
    std::vector<int> parent;        // front, -1 at a root
    std::vector<int> idx_ptr, idx;  // the front's nodes (global columns: pivots then rows), ascending
    std::vector<int> cmap;          // per front, at idx_ptr + npiv: its rows' places in its parent's node list
    std::vector<int> child_ptr, child;
    std::vector<int> level_ptr;     // fronts of level L: [level_ptr[L], level_ptr[L + 1])
    std::vector<int> comp;          // the component each front belongs to (global)
    double flops = 0;               // per factorization (multiply and add counted apart)
    double entries = 0;             // dense lower-triangle entries over all fronts (DOF^2 / 2)
};

struct MfParams { // relaxed amalgamation, in frame nodes (CHOLMOD's rule of thumb, scaled to 6 x 6 blocks)
    int small = 4;        // merged groups up to this many columns merge whatever their zeros
    int mid = 16;         // ... up to this many, while zeros stay under mid_frac of the entries
    double mid_frac = 0.5;
    int large = 48;
    double large_frac = 0.1;
    double huge_frac = 0.05;
};

// the columns [0, n) of the pattern col_ptr / row (rows ascending; comp_of_col: each column's component): the fronts'
// columns, their top columns and components appended to fr_cols / fr_top / fr_comp
static void mf_plan_columns(int n, const std::vector<int>& col_ptr, const std::vector<int>& row, const std::vector<int>& comp_of_col,
                            std::vector<std::vector<int>>& fr_cols, std::vector<int>& fr_top, std::vector<int>& fr_comp,
                            const MfParams& prm = MfParams{}) {
    std::vector<int> parent(n, -1), nchild(n, 0), only_child(n, -1);
    for (int k = 0; k < n; k++)
        if (col_ptr[k + 1] > col_ptr[k]) {
            parent[k] = row[col_ptr[k]];
            nchild[parent[k]]++, only_child[parent[k]] = k;
        }
    // fundamental supernodes: groups of columns, each in ascending order
    std::vector<int> group(n, -1);
    std::vector<std::vector<int>> cols;
    std::vector<int> top; // the group's last column (its structure is the group's rows)
    for (int k = 0; k < n; k++) {
        const int c = only_child[k];
        const bool chain = nchild[k] == 1 && (col_ptr[c + 1] - col_ptr[c]) == (col_ptr[k + 1] - col_ptr[k]) + 1;
        if (chain) {
            group[k] = group[c];
            cols[group[k]].push_back(k);
            top[group[k]] = k;
        } else {
            group[k] = (int)cols.size();
            cols.push_back({k});
            top.push_back(k);
        }
    }
    const int G = (int)cols.size();
    // the group tree; groups in order of their top column come children before parents
    std::vector<int> gpar(G, -1);
    for (int g = 0; g < G; g++)
        if (parent[top[g]] >= 0) gpar[g] = group[parent[top[g]]];
    std::vector<int> gorder(G);
    for (int g = 0; g < G; g++) gorder[g] = g;
    std::sort(gorder.begin(), gorder.end(), [&](int a, int b) { return top[a] < top[b]; });
    // relaxed amalgamation: zeros[g] / entries[g] over the group's columns in the front it would form
    std::vector<double> zeros(G, 0.0), entries(G, 0.0);
    std::vector<int> alive(G, 1), merged_into(G, -1);
    auto nrows = [&](int g) { return col_ptr[top[g] + 1] - col_ptr[top[g]]; };
    for (int g = 0; g < G; g++) {
        const double m = (double)cols[g].size(), r = nrows(g);
        entries[g] = m * (m + 1) / 2 + m * r;
    }
    auto root_of = [&](int g) {
        while (merged_into[g] >= 0) g = merged_into[g];
        return g;
    };
    for (int gi = 0; gi < G; gi++) {
        const int s = gorder[gi];
        if (gpar[s] < 0) continue;
        const int p = root_of(gpar[s]);
        const double ms = (double)cols[s].size(), mp = (double)cols[p].size(), rp = nrows(p), rs = nrows(s);
        // S's columns in the merged front reach P's columns and rows instead of their own rows
        const double added = ms * (mp + rp - rs);
        const double z = zeros[s] + zeros[p] + added, e = entries[s] + entries[p] + added;
        const double mm = ms + mp, frac = z / e;
        const bool take = mm <= prm.small || (mm <= prm.mid && frac < prm.mid_frac) || (mm <= prm.large && frac < prm.large_frac) || frac < prm.huge_frac;
        if (!take) continue;
        for (int k : cols[s]) cols[p].push_back(k);
        std::vector<int>().swap(cols[s]);
        zeros[p] = z, entries[p] = e;
        alive[s] = 0, merged_into[s] = p;
    }
    for (int g = 0; g < G; g++) {
        if (!alive[g]) continue;
        std::sort(cols[g].begin(), cols[g].end());
        fr_cols.push_back(cols[g]);
        fr_top.push_back(top[g]);
        fr_comp.push_back(comp_of_col[cols[g][0]]);
    }
}

// the fronts (their columns) into the plan: rows, tree, levels, maps
static MfPlan mf_finish(int NF, const std::vector<int>& col_ptr, const std::vector<int>& row, const std::vector<std::vector<int>>& fr_cols,
                        const std::vector<int>& fr_top, const std::vector<int>& fr_comp) {
    MfPlan P;
    const int nfr = (int)fr_cols.size();
    std::vector<int> front_of(NF, -1);
    for (int f = 0; f < nfr; f++)
        for (int k : fr_cols[f]) front_of[k] = f;
    std::vector<int> fpar(nfr, -1), lvl(nfr, 0);
    for (int f = 0; f < nfr; f++) {
        const int t = fr_top[f];
        if (col_ptr[t + 1] > col_ptr[t]) fpar[f] = front_of[row[col_ptr[t]]];
    }
    // levels: a front one above its highest child (children have lower top columns: one pass in top order)
    std::vector<int> order(nfr);
    for (int f = 0; f < nfr; f++) order[f] = f;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return fr_top[a] < fr_top[b]; });
    for (int f : order)
        if (fpar[f] >= 0) lvl[fpar[f]] = std::max(lvl[fpar[f]], lvl[f] + 1);
    int nlev = 0;
    for (int f = 0; f < nfr; f++) nlev = std::max(nlev, lvl[f] + 1);
    // execution order: by level, then by size (largest first, so the long blocks start early), then by top column
    std::vector<int> ex(nfr);
    for (int f = 0; f < nfr; f++) ex[f] = f;
    auto rows_of = [&](int f) { return col_ptr[fr_top[f] + 1] - col_ptr[fr_top[f]]; };
    std::sort(ex.begin(), ex.end(), [&](int a, int b) {
        if (lvl[a] != lvl[b]) return lvl[a] < lvl[b];
        const int sa = (int)fr_cols[a].size() + rows_of(a), sb = (int)fr_cols[b].size() + rows_of(b);
        if (sa != sb) return sa > sb;
        return fr_top[a] < fr_top[b];
    });
    std::vector<int> pos(nfr);
    for (int i = 0; i < nfr; i++) pos[ex[i]] = i;
    P.level_ptr.assign(nlev + 1, 0);
    for (int f = 0; f < nfr; f++) P.level_ptr[lvl[f] + 1]++;
    for (int L = 0; L < nlev; L++) P.level_ptr[L + 1] += P.level_ptr[L];
    P.idx_ptr.assign(1, 0);
    for (int i = 0; i < nfr; i++) {
        const int f = ex[i];
        const int t = fr_top[f];
        P.npiv.push_back((int)fr_cols[f].size());
        P.nrow.push_back(col_ptr[t + 1] - col_ptr[t]);
        P.parent.push_back(fpar[f] >= 0 ? pos[fpar[f]] : -1);
        P.comp.push_back(fr_comp[f]);
        P.idx.insert(P.idx.end(), fr_cols[f].begin(), fr_cols[f].end());
        P.idx.insert(P.idx.end(), row.begin() + col_ptr[t], row.begin() + col_ptr[t + 1]);
        P.idx_ptr.push_back((int)P.idx.size());
        const double p = 6.0 * P.npiv.back(), r = 6.0 * P.nrow.back();
        P.flops += p * p * p / 3 + p * p * r + p * r * r;
        P.entries += (p + r) * (p + r + 1) / 2;
    }
    // each front's rows in its parent's node list (both ascending: one merge walk)
    P.cmap.assign(P.idx.size(), -1);
    for (int f = 0; f < nfr; f++) {
        const int q = P.parent[f];
        if (q < 0) continue;
        int a = P.idx_ptr[q];
        for (int x = P.idx_ptr[f] + P.npiv[f]; x < P.idx_ptr[f + 1]; x++) {
            while (a < P.idx_ptr[q + 1] && P.idx[a] < P.idx[x]) a++;
            P.cmap[x] = a - P.idx_ptr[q]; // (always found: a front's rows are in its parent's list)
        }
    }
    // children in execution order
    std::vector<std::vector<int>> ch(nfr);
    for (int f = 0; f < nfr; f++)
        if (P.parent[f] >= 0) ch[P.parent[f]].push_back(f);
    P.child_ptr.assign(1, 0);
    for (int f = 0; f < nfr; f++) {
        P.child.insert(P.child.end(), ch[f].begin(), ch[f].end());
        P.child_ptr.push_back((int)P.child.size());
    }
    return P;
}

} // namespace blg
