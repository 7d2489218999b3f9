// The reference's sequential orderings: incidence degree (ID), saturation degree (SD) and its
// batched variant (SDA), src/incidence_degree.c:107-361.  They pick one vertex at a time by a
// running count that depends on every earlier pick, so they stay on the host; the library exports
// them under the reference's names so that its quick mode (src/main.c:135-188) and callers that
// link the reference's main.c find them here.
//
// Selection rule (incidence_degree.c:7-14): the next vertex is the top of a binary heap ordered by
// count, then degree, then id (largest first); see Queue for why the heap itself is reproduced.
//
// Growth (ID, SD): the first component processed is vertex 0's, started from its maximum-degree
// vertex (the first such vertex by id).  A neighbour enters the queue when its count first changes.
// When the queue empties, the scan over vertex ids k = 0, 1, ... starts the component of the next
// vertex k that has no priority yet; a component first reached at the last id is therefore never
// processed and keeps p = -1, as in the reference's loop (incidence_degree.c:132-157).
//
// SD (incidence_degree.c:166-255): each picked vertex takes the first color free among its
// neighbours; an uncolored neighbour's count grows when that color is new among its colored
// neighbours, i.e. the count is the number of distinct neighbour colors (the reference rescans the
// neighbour's list; a per-vertex set of seen colors gives the same counts in O(degree)).
//
// SDA (incidence_degree.c:257-361): every vertex whose degree equals its component's maximum starts
// in the queue; all queue-top vertices with the same (count, degree) as the top are picked together
// and share one priority, then colored in pick order.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "incidence_degree.h"

namespace {

// The reference's priority queue, operation for operation: a 1-based binary max-heap over
// (count, degree, id) with a position index per vertex.  Insert sifts up; removing slot i moves the
// last entry there and sifts *down* only.  Removing a slot from the middle can therefore leave an
// entry above a smaller parent, and the later picks follow the resulting heap, not the true
// maximum: the orderings depend on these exact mechanics (incidence_degree.c:16-73), so they are
// reproduced rather than replaced by another max-structure.
struct Queue {
    std::vector<uint32_t> heap, pos;  // heap[1..n]; pos[u] = slot of u, 0 when absent
    uint32_t n = 0;
    const std::vector<uint32_t> &count;
    const uint32_t *V;
    Queue(uint32_t N, const std::vector<uint32_t> &c, const uint32_t *V_)
        : heap((size_t)N + 2, UINT32_MAX), pos(N, 0), count(c), V(V_) {}
    bool above(uint32_t a, uint32_t b) const {  // a belongs above b
        if (count[a] != count[b]) return count[a] > count[b];
        const uint32_t da = V[a + 1] - V[a], db = V[b + 1] - V[b];
        if (da != db) return da > db;
        return a > b;
    }
    void place(uint32_t slot, uint32_t u) {
        heap[slot] = u;
        pos[u] = slot;
    }
    void insert(uint32_t u) {
        uint32_t i = ++n;
        place(i, u);
        while (i != 1 && above(u, heap[i >> 1])) {
            place(i, heap[i >> 1]);
            i >>= 1;
            place(i, u);
        }
    }
    void sift_down(uint32_t i) {
        for (;;) {
            const uint32_t l = 2 * i, r = 2 * i + 1;
            uint32_t m = i;
            if (l <= n && above(heap[l], heap[m])) m = l;
            if (r <= n && above(heap[r], heap[m])) m = r;
            if (m == i) return;
            const uint32_t x = heap[i], y = heap[m];
            place(i, y);
            place(m, x);
            i = m;
        }
    }
    void remove_slot(uint32_t i) {
        if (i == 0) return;
        const uint32_t x = heap[i], y = heap[n];
        place(i, y);
        heap[n] = UINT32_MAX;
        pos[x] = 0;
        n--;
        sift_down(i);
    }
    // the count of u changed (or u is new): out of its slot, back in from the bottom
    void put(uint32_t u) {
        remove_slot(pos[u]);
        insert(u);
    }
    uint32_t top() const { return heap[1]; }
    uint32_t pop() {
        const uint32_t u = heap[1];
        remove_slot(1);
        return u;
    }
    bool empty() const { return n == 0; }
};

// Component labels (iterative: the reference's recursive walk overflows the stack on large graphs).
std::vector<uint32_t> components(uint32_t N, const uint32_t *V, const uint32_t *E, uint32_t *n_cc) {
    std::vector<uint32_t> cc(N, UINT32_MAX), stack;
    uint32_t t = 0;
    for (uint32_t s = 0; s < N; s++) {
        if (cc[s] != UINT32_MAX) continue;
        cc[s] = t;
        stack.push_back(s);
        while (!stack.empty()) {
            const uint32_t u = stack.back();
            stack.pop_back();
            for (uint32_t i = V[u]; i < V[u + 1]; i++)
                if (cc[E[i]] == UINT32_MAX) {
                    cc[E[i]] = t;
                    stack.push_back(E[i]);
                }
        }
        t++;
    }
    *n_cc = t;
    return cc;
}

// First vertex (by id) of maximum degree in each component.
std::vector<uint32_t> component_starts(uint32_t N, const uint32_t *V, const std::vector<uint32_t> &cc, uint32_t n_cc) {
    std::vector<uint32_t> md(n_cc, UINT32_MAX);
    for (uint32_t u = 0; u < N; u++) {
        uint32_t &m = md[cc[u]];
        if (m == UINT32_MAX || V[m + 1] - V[m] < V[u + 1] - V[u]) m = u;
    }
    return md;
}

// First color >= 1 that no neighbour of u has.
int first_free(uint32_t u, const uint32_t *V, const uint32_t *E, const std::vector<int> &color,
               std::vector<uint32_t> &mark) {
    for (uint32_t i = V[u]; i < V[u + 1]; i++) mark[color[E[i]]] = u;
    int c = 1;
    while (mark[c] == u) c++;
    return c;
}

// Adds color c to v's seen colors; true when it was new.
bool see(std::vector<std::vector<uint32_t>> &seen, uint32_t v, uint32_t c) {
    auto &s = seen[v];
    if (std::find(s.begin(), s.end(), c) != s.end()) return false;
    s.push_back(c);
    return true;
}

// ID and SD share the growth loop; `pick` handles one picked vertex.
template <class Pick>
void grow(uint32_t N, const uint32_t *V, const uint32_t *E, double *p, Queue &q, Pick pick) {
    uint32_t n_cc = 0;
    const std::vector<uint32_t> cc = components(N, V, E, &n_cc);
    const std::vector<uint32_t> md = component_starts(N, V, cc, n_cc);
    for (uint32_t u = 0; u < N; u++) p[u] = -1.0;
    double t = (double)N;
    q.put(md[cc[0]]);
    for (uint32_t k = 0; k < N; k++) {
        while (!q.empty()) {
            const uint32_t u = q.pop();
            p[u] = t;
            t -= 1.0;
            pick(u);
        }
        if (p[k] < 0.0) q.put(md[cc[k]]);  // a component reached at the last id is never drained
    }
}

}  // namespace

extern "C" {

void incidence_degree_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p) {
    if (N == 0) return;
    std::vector<uint32_t> count(N, 0);
    Queue q(N, count, V);
    grow(N, V, E, p, q, [&](uint32_t u) {
        for (uint32_t i = V[u]; i < V[u + 1]; i++) {
            const uint32_t v = E[i];
            if (p[v] >= 0.0) continue;
            count[v]++;
            q.put(v);
        }
    });
}

void saturation_degree_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p) {
    if (N == 0) return;
    std::vector<uint32_t> count(N, 0), mark((size_t)N + 2, UINT32_MAX);
    std::vector<int> color(N, 0);
    std::vector<std::vector<uint32_t>> seen(N);
    Queue q(N, count, V);
    grow(N, V, E, p, q, [&](uint32_t u) {
        const int c = first_free(u, V, E, color, mark);
        color[u] = c;
        for (uint32_t i = V[u]; i < V[u + 1]; i++) {
            const uint32_t v = E[i];
            if (p[v] >= 0.0) continue;
            if (see(seen, v, (uint32_t)c)) {
                count[v]++;
                q.put(v);
            }
        }
    });
}

void saturation_degree_ordering_alt(uint32_t N, const uint32_t *V, const uint32_t *E, double *p) {
    if (N == 0) return;
    uint32_t n_cc = 0;
    const std::vector<uint32_t> cc = components(N, V, E, &n_cc);
    std::vector<uint32_t> maxdeg(n_cc, 0);
    for (uint32_t u = 0; u < N; u++) maxdeg[cc[u]] = std::max(maxdeg[cc[u]], V[u + 1] - V[u]);
    std::vector<uint32_t> count(N, 0), mark((size_t)N + 2, UINT32_MAX), batch;
    std::vector<int> color(N, 0);
    std::vector<std::vector<uint32_t>> seen(N);
    Queue q(N, count, V);
    for (uint32_t u = 0; u < N; u++) p[u] = -1.0;
    for (uint32_t u = 0; u < N; u++)
        if (V[u + 1] - V[u] == maxdeg[cc[u]]) q.put(u);
    double t = (double)N;
    while (!q.empty()) {
        const uint32_t best = q.top();
        const uint32_t best_count = count[best], best_deg = V[best + 1] - V[best];
        batch.clear();
        while (!q.empty() && count[q.top()] == best_count && V[q.top() + 1] - V[q.top()] == best_deg) {
            const uint32_t u = q.pop();
            p[u] = t;
            batch.push_back(u);
        }
        t -= 1.0;
        for (uint32_t u : batch) {
            const int c = first_free(u, V, E, color, mark);
            color[u] = c;
            for (uint32_t i = V[u]; i < V[u + 1]; i++) {
                const uint32_t v = E[i];
                if (p[v] >= 0.0) continue;
                if (see(seen, v, (uint32_t)c)) {
                    count[v]++;
                    q.put(v);
                }
            }
        }
    }
}

}  // extern "C"
