#include "chol_symbolic.h"

#include <algorithm>
#include <cmath>
#include <functional>
#include <numeric>

namespace efem {

namespace {

constexpr int kLeaf = 40;  // parts at or below this size are not dissected further

// Geometric nested dissection: split a part at the median coordinate of its
// longest bounding-box axis; the smaller of the two boundary layers becomes
// the vertex separator, ordered after both halves.
void dissect(std::vector<int>& part, const std::vector<int>& rp, const std::vector<int>& ci, const double* X,
    std::vector<signed char>& side, std::vector<int>& order)
{
    if (static_cast<int>(part.size()) <= kLeaf) {
        std::sort(part.begin(), part.end());
        order.insert(order.end(), part.begin(), part.end());
        return;
    }
    double lo[3] = { 1e300, 1e300, 1e300 }, hi[3] = { -1e300, -1e300, -1e300 };
    for (int v : part)
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], X[3 * v + k]);
            hi[k] = std::max(hi[k], X[3 * v + k]);
        }
    int ax = 0;
    for (int k = 1; k < 3; k++)
        if (hi[k] - lo[k] > hi[ax] - lo[ax]) ax = k;
    std::vector<int> srt(part);
    const size_t mid = srt.size() / 2;
    std::nth_element(srt.begin(), srt.begin() + mid, srt.end(),
        [&](int a, int b) { return X[3 * a + ax] < X[3 * b + ax] || (X[3 * a + ax] == X[3 * b + ax] && a < b); });
    const double m = X[3 * srt[mid] + ax];
    std::vector<int> L, R;
    for (int v : part) (X[3 * v + ax] < m ? L : R).push_back(v);
    if (L.empty() || R.empty()) {  // all on one plane: split by rank
        L.assign(srt.begin(), srt.begin() + mid);
        R.assign(srt.begin() + mid, srt.end());
    }
    for (int v : L) side[v] = 0;
    for (int v : R) side[v] = 1;
    std::vector<int> SL, SR;
    auto touches = [&](int v, int other) {
        for (int k = rp[v]; k < rp[v + 1]; k++)
            if (side[ci[k]] == other) return true;
        return false;
    };
    for (int v : L)
        if (touches(v, 1)) SL.push_back(v);
    for (int v : R)
        if (touches(v, 0)) SR.push_back(v);
    std::vector<int>& S = SL.size() <= SR.size() ? SL : SR;
    std::vector<int>& from = SL.size() <= SR.size() ? L : R;
    for (int v : S) side[v] = 2;
    from.erase(std::remove_if(from.begin(), from.end(), [&](int v) { return side[v] == 2; }), from.end());
    for (int v : part) side[v] = -1;
    std::vector<int> Sk(S);
    std::vector<int>().swap(part);
    dissect(L, rp, ci, X, side, order);
    dissect(R, rp, ci, X, side, order);
    std::sort(Sk.begin(), Sk.end());
    order.insert(order.end(), Sk.begin(), Sk.end());
}

}  // namespace

void symbolic_analysis(int n, const std::vector<int>& rowptr, const std::vector<int>& col, const double* coords,
    Symbolic& S)
{
    S = Symbolic();
    S.n = n;
    if (n == 0) return;
    // ---------------------------------------------------------------- ordering
    std::vector<int> order;
    order.reserve(n);
    {
        std::vector<int> all(n);
        std::iota(all.begin(), all.end(), 0);
        std::vector<signed char> side(n, -1);
        dissect(all, rowptr, col, coords, side, order);
    }
    std::vector<int> perm = order, iperm(n);
    for (int i = 0; i < n; i++) iperm[perm[i]] = i;

    // ---------------------------------------------------------------- elimination tree (Liu)
    auto etree = [&](const std::vector<int>& pm, const std::vector<int>& ipm, std::vector<int>& par) {
        par.assign(n, -1);
        std::vector<int> anc(n, -1);
        for (int j = 0; j < n; j++) {
            const int o = pm[j];
            for (int k = rowptr[o]; k < rowptr[o + 1]; k++) {
                int i = ipm[col[k]];
                if (i >= j) continue;
                while (anc[i] != -1 && anc[i] != j) {
                    const int t = anc[i];
                    anc[i] = j;
                    i = t;
                }
                if (anc[i] == -1) {
                    anc[i] = j;
                    par[i] = j;
                }
            }
        }
    };
    std::vector<int> par;
    etree(perm, iperm, par);
    // postorder so that every subtree is a contiguous range of columns
    {
        std::vector<int> head(n, -1), next(n, -1);
        for (int j = n - 1; j >= 0; j--)
            if (par[j] >= 0) {
                next[j] = head[par[j]];
                head[par[j]] = j;
            }
        std::vector<int> post;
        post.reserve(n);
        std::vector<int> stack;
        for (int r = 0; r < n; r++) {
            if (par[r] != -1) continue;
            stack.push_back(r);
            while (!stack.empty()) {
                const int v = stack.back();
                if (head[v] != -1) {
                    const int c = head[v];
                    head[v] = next[c];
                    stack.push_back(c);
                } else {
                    stack.pop_back();
                    post.push_back(v);
                }
            }
        }
        std::vector<int> np(n);
        for (int k = 0; k < n; k++) np[k] = perm[post[k]];
        perm.swap(np);
        for (int i = 0; i < n; i++) iperm[perm[i]] = i;
        etree(perm, iperm, par);
    }
    S.perm = perm;
    S.iperm = iperm;

    // ---------------------------------------------------------------- column structures
    std::vector<std::vector<int>> kids(n);
    for (int j = 0; j < n; j++)
        if (par[j] >= 0) kids[par[j]].push_back(j);
    std::vector<std::vector<int>> st(n);
    std::vector<int> cnt(n, 0), mark(n, -1);
    // supernode (fundamental) bookkeeping
    std::vector<int> sfirst, sncol;
    std::vector<std::vector<int>> sbelow;  // below rows of each supernode's last column
    for (int j = 0; j < n; j++) {
        std::vector<int> s;
        mark[j] = j;
        const int o = perm[j];
        for (int k = rowptr[o]; k < rowptr[o + 1]; k++) {
            const int i = iperm[col[k]];
            if (i > j && mark[i] != j) {
                mark[i] = j;
                s.push_back(i);
            }
        }
        for (int c : kids[j])
            for (int i : st[c])
                if (i != j && mark[i] != j) {
                    mark[i] = j;
                    s.push_back(i);
                }
        std::sort(s.begin(), s.end());
        cnt[j] = static_cast<int>(s.size());
        const bool cont = j > 0 && par[j - 1] == j && kids[j].size() == 1 && cnt[j - 1] == cnt[j] + 1;
        if (!cont) {
            if (j > 0) sbelow.push_back(st[j - 1]);  // close the previous supernode
            sfirst.push_back(j);
            sncol.push_back(1);
        } else {
            sncol.back()++;
        }
        for (int c : kids[j]) std::vector<int>().swap(st[c]);
        st[j].swap(s);
    }
    sbelow.push_back(st[n - 1]);
    std::vector<std::vector<int>>().swap(st);

    // ---------------------------------------------------------------- relaxed amalgamation
    int nsf = static_cast<int>(sfirst.size());
    std::vector<int> snode_of(n);
    for (int s = 0; s < nsf; s++)
        for (int k = 0; k < sncol[s]; k++) snode_of[sfirst[s] + k] = s;
    std::vector<int> sparent(nsf, -1);
    for (int s = 0; s < nsf; s++)
        if (!sbelow[s].empty()) sparent[s] = snode_of[sbelow[s][0]];
    std::vector<int> alias(nsf);
    std::iota(alias.begin(), alias.end(), 0);
    std::function<int(int)> find = [&](int s) { return alias[s] == s ? s : alias[s] = find(alias[s]); };
    std::vector<char> alive(nsf, 1);
    auto nnz_of = [](long long c, long long r) { return c * r - c * (c - 1) / 2; };
    for (bool changed = true; changed;) {  // repeat: a merge exposes a new rightmost child
        changed = false;
        for (int s = 0; s < nsf; s++) {
            if (!alive[s] || sparent[s] < 0) continue;
            const int p = find(sparent[s]);
            if (sfirst[s] + sncol[s] != sfirst[p]) continue;  // not the child right before the parent
            const long long cs = sncol[s], rs = cs + static_cast<long long>(sbelow[s].size());
            const long long cp = sncol[p], rpn = cp + static_cast<long long>(sbelow[p].size());
            const long long c = cs + cp, r = cs + rpn;
            const long long zeros = nnz_of(c, r) - nnz_of(cs, rs) - nnz_of(cp, rpn);
            const double frac = static_cast<double>(zeros) / static_cast<double>(nnz_of(c, r));
            const bool merge = c <= 4 || (c <= 16 && frac < 0.8) || (c <= 48 && frac < 0.1) || frac < 0.05;
            if (!merge) continue;
            sfirst[p] = sfirst[s];
            sncol[p] += sncol[s];
            alive[s] = 0;
            alias[s] = p;
            changed = true;
        }
    }
    // surviving supernodes, in column order
    std::vector<int> ids;
    for (int s = 0; s < nsf; s++)
        if (alive[s]) ids.push_back(s);
    std::sort(ids.begin(), ids.end(), [&](int a, int b) { return sfirst[a] < sfirst[b]; });
    const int ns = static_cast<int>(ids.size());
    S.ns = ns;
    std::vector<int> newid(nsf, -1);
    for (int k = 0; k < ns; k++) newid[ids[k]] = k;
    S.first.resize(ns);
    S.ncol.resize(ns);
    S.nrow.resize(ns);
    S.rows_off.resize(ns + 1);
    S.rows_off[0] = 0;
    for (int k = 0; k < ns; k++) {
        const int s = ids[k];
        S.first[k] = sfirst[s];
        S.ncol[k] = sncol[s];
        // rows: own columns, then the below rows of the (merged) last column
        for (int c = 0; c < sncol[s]; c++) S.rows.push_back(sfirst[s] + c);
        for (int i : sbelow[s]) S.rows.push_back(i);
        S.nrow[k] = sncol[s] + static_cast<int>(sbelow[s].size());
        S.rows_off[k + 1] = static_cast<long long>(S.rows.size());
    }
    std::vector<int> front_of(n);
    for (int k = 0; k < ns; k++)
        for (int c = 0; c < S.ncol[k]; c++) front_of[S.first[k] + c] = k;
    S.parent.assign(ns, -1);
    for (int k = 0; k < ns; k++)
        if (S.nrow[k] > S.ncol[k]) S.parent[k] = front_of[S.rows[S.rows_off[k] + S.ncol[k]]];
    // children lists (increasing order) and levels
    S.child_ptr.assign(ns + 1, 0);
    for (int k = 0; k < ns; k++)
        if (S.parent[k] >= 0) S.child_ptr[S.parent[k] + 1]++;
    for (int k = 0; k < ns; k++) S.child_ptr[k + 1] += S.child_ptr[k];
    S.child_list.resize(S.child_ptr[ns]);
    {
        std::vector<int> fill(ns, 0);
        for (int k = 0; k < ns; k++)
            if (S.parent[k] >= 0) S.child_list[S.child_ptr[S.parent[k]] + fill[S.parent[k]]++] = k;
    }
    std::vector<int> level(ns, 0);
    int nlev = 0;
    for (int k = 0; k < ns; k++) {  // children precede parents
        if (S.parent[k] >= 0) level[S.parent[k]] = std::max(level[S.parent[k]], level[k] + 1);
        nlev = std::max(nlev, level[k] + 1);
    }
    S.level_ptr.assign(nlev + 1, 0);
    for (int k = 0; k < ns; k++) S.level_ptr[level[k] + 1]++;
    for (int l = 0; l < nlev; l++) S.level_ptr[l + 1] += S.level_ptr[l];
    S.level_list.resize(ns);
    {
        std::vector<int> fill(nlev, 0);
        for (int k = 0; k < ns; k++) S.level_list[S.level_ptr[level[k]] + fill[level[k]]++] = k;
    }
    // relative indices of each front's below rows inside its parent's rows
    S.relind_off.assign(ns + 1, 0);
    for (int k = 0; k < ns; k++) {
        S.relind_off[k + 1] = S.relind_off[k];
        if (S.parent[k] < 0) continue;
        const int p = S.parent[k];
        const int* pr = S.rows.data() + S.rows_off[p];
        const int pn = S.nrow[p];
        int q = 0;
        for (int a = S.ncol[k]; a < S.nrow[k]; a++) {
            const int row = S.rows[S.rows_off[k] + a];
            while (q < pn && pr[q] < row) q++;
            S.relind.push_back(q);  // pr[q] == row by the elimination-tree property
        }
        S.relind_off[k + 1] = static_cast<long long>(S.relind.size());
    }
    // storage offsets and flop count
    S.front_off.resize(ns + 1);
    S.dinv_off.resize(ns + 1);
    S.upd_off.resize(ns + 1);
    S.lt_off.resize(ns + 1);
    S.front_off[0] = S.dinv_off[0] = S.upd_off[0] = S.lt_off[0] = 0;
    S.nnz_L = 0;
    S.flops = 0;
    for (int k = 0; k < ns; k++) {
        const long long r = S.nrow[k], c = S.ncol[k];
        S.front_off[k + 1] = S.front_off[k] + r * r;
        S.dinv_off[k + 1] = S.dinv_off[k] + c * c;
        S.upd_off[k + 1] = S.upd_off[k] + 3 * (r - c);
        S.lt_off[k + 1] = S.lt_off[k] + (r - c) * c;
        S.nnz_L += c * r - c * (c - 1) / 2;
        S.flops += c * c * c / 3.0 + static_cast<double>(r - c) * c * c + static_cast<double>(r - c) * (r - c) * c;
    }
    S.front_size = S.front_off[ns];
    S.dinv_size = S.dinv_off[ns];
    S.upd_size = S.upd_off[ns];
    S.lt_size = S.lt_off[ns];
    // children's update-vector entries per parent row, in child order
    {
        std::vector<int> cnt(S.rows.size() + 1, 0);
        for (int k = 0; k < ns; k++) {
            if (S.parent[k] < 0) continue;
            const long long base = S.rows_off[S.parent[k]];
            for (long long j = S.relind_off[k]; j < S.relind_off[k + 1]; j++) cnt[base + S.relind[j] + 1]++;
        }
        for (size_t i = 0; i + 1 < cnt.size(); i++) cnt[i + 1] += cnt[i];
        S.contrib_ptr = cnt;
        S.below_front.assign(static_cast<size_t>(S.upd_size / 3), 0);
        for (int k = 0; k < ns; k++)
            for (long long q = S.upd_off[k] / 3; q < S.upd_off[k + 1] / 3; q++) S.below_front[q] = k;
        S.contrib_idx.assign(cnt.back(), 0);
        std::vector<int> fill(S.rows.size(), 0);
        for (int s = 0; s < ns; s++)  // parents in order, children in list order
            for (int q = S.child_ptr[s]; q < S.child_ptr[s + 1]; q++) {
                const int ch = S.child_list[q];
                const long long base = S.rows_off[s];
                for (long long j = S.relind_off[ch]; j < S.relind_off[ch + 1]; j++) {
                    const long long row = base + S.relind[j];
                    S.contrib_idx[S.contrib_ptr[row] + fill[row]++] =
                        static_cast<int>(S.upd_off[ch] / 3 + (j - S.relind_off[ch]));
                }
            }
    }
    // original entries (lower triangle) -> front positions
    for (int o = 0; o < n; o++) {
        const int j = iperm[o];
        const int k = front_of[j];
        const int* rr = S.rows.data() + S.rows_off[k];
        const int r = S.nrow[k];
        const long long colbase = S.front_off[k] + static_cast<long long>(j - S.first[k]) * r;
        for (int e = rowptr[o]; e < rowptr[o + 1]; e++) {
            const int i = iperm[col[e]];
            if (i < j) continue;
            const int pos = static_cast<int>(std::lower_bound(rr, rr + r, i) - rr);
            S.a_pos.push_back(colbase + pos);
            S.a_src.push_back(e);
        }
    }
}

}  // namespace efem
