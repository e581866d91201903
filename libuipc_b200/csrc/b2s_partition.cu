// Graph partition of a mesh's vertex adjacency into parts of at most
// max_part vertices: the caller-side step geometry::mesh_partition performs
// with METIS k-way before FEMMASPreconditioner::do_init
// (src/geometry/mesh_partition.cpp:77-231: ceil(n / max_part) parts of at most
// max_part vertices from connectivity alone; point clouds fall back to
// sequential blocks).
//
// Design: recursive graph bisection, depth first with the left side first, so
// that part ids follow the bisection tree and consecutive parts are graph
// neighbours (the MAS hierarchy groups 16 consecutive parts into one bank of
// the next level). Every left side holds whole parts: a range of m vertices
// (p = ceil(m / max_part) parts) keeps ceil(p / 2) * max_part on the left, so
// a range's first vertex index is a multiple of max_part and its part ids are
// fixed by its position alone, whatever order the subtrees run in.
//
// One bisection:
//  1. seed: a pseudo-peripheral vertex (two breadth-first sweeps inside the
//     range from its lowest-numbered vertex);
//  2. growth: the left side grows from the seed by always taking the frontier
//     vertex with the largest gain (edges into the side minus edges to the
//     rest of the range; ties to the earliest discovered), restarting from
//     the first unreached vertex when a component is used up;
//  3. refinement: balanced swaps of a left and a right boundary vertex while
//     the pair lowers the cut (gain_a + gain_b - 2 [a ~ b] > 0), each vertex
//     moved once per pass, a few passes.
// Membership of a neighbour in the range being split is read from a tag array
// (the range's first index); ranges that run concurrently hold disjoint tags.
#include "b2s_internal.cuh"

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <future>
#include <queue>
#include <vector>

namespace b2s
{
namespace
{
struct PartGraph
{
    int32_t                              n;
    const int32_t*                       xadj;
    const int32_t*                       adj;
    int32_t                              max_part;
    std::vector<int32_t>                 order;  // ranges of this array are the subsets
    std::vector<std::atomic<int32_t>>    tag;    // first index of the vertex's current range
    int32_t*                             part_ids;

    bool inside(int32_t u, int32_t lo) const { return tag[u].load(std::memory_order_relaxed) == lo; }
};

constexpr int REFINE_PASSES = 4;
constexpr int PARALLEL_DEPTH = 5;  // up to 32 concurrent subtrees

// vertices of the range reached from `src` in breadth-first order; returns the last
int32_t bfs_far(const PartGraph& G, int32_t lo, int32_t src, std::vector<int32_t>& dist,
                std::vector<int32_t>& queue)
{
    queue.clear();
    queue.push_back(src);
    dist[src]    = 0;
    size_t head  = 0;
    int32_t last = src;
    while(head < queue.size())
    {
        const int32_t v = queue[head++];
        last            = v;
        for(int32_t e = G.xadj[v]; e < G.xadj[v + 1]; ++e)
        {
            const int32_t u = G.adj[e];
            if(u == v || !G.inside(u, lo) || dist[u] >= 0)
                continue;
            dist[u] = dist[v] + 1;
            queue.push_back(u);
        }
    }
    for(int32_t v : queue)
        dist[v] = -1;
    return last;
}

struct Cand
{
    int32_t gain;
    int32_t order;  // discovery order: earlier first among equal gains
    int32_t v;
    bool    operator<(const Cand& o) const { return gain < o.gain || (gain == o.gain && order > o.order); }
};

// side[v]: 0 left, 1 right, for the vertices of [lo, hi); per-vertex scratch
// arrays are indexed by global vertex id and restored to their idle values.
struct Scratch
{
    std::vector<int32_t> dist;   // -1 idle
    std::vector<int32_t> gain;   // growth: edges into left minus edges to the rest
    std::vector<int8_t>  state;  // 0 idle/unreached, 1 frontier, 2 taken (growth); moved flag (refine)
    std::vector<int8_t>  side;
    std::vector<int32_t> queue;
    explicit Scratch(int32_t n) : dist(n, -1), gain(n, 0), state(n, 0), side(n, 0) {}
};

void grow_left(const PartGraph& G, int32_t lo, int32_t hi, int32_t want, Scratch& S)
{
    const int32_t* W = G.order.data();
    for(int32_t k = lo; k < hi; ++k)
        S.side[W[k]] = 1;
    // pseudo-peripheral seed from the range's lowest-numbered vertex
    int32_t first = W[lo];
    for(int32_t k = lo + 1; k < hi; ++k)
        first = std::min(first, W[k]);
    const int32_t a    = bfs_far(G, lo, first, S.dist, S.queue);
    const int32_t seed = bfs_far(G, lo, a, S.dist, S.queue);

    std::priority_queue<Cand> pq;
    int32_t taken = 0, stamp = 0, scan = lo;
    auto take = [&](int32_t v)
    {
        S.state[v] = 2;
        S.side[v]  = 0;
        ++taken;
        for(int32_t e = G.xadj[v]; e < G.xadj[v + 1]; ++e)
        {
            const int32_t u = G.adj[e];
            if(u == v || !G.inside(u, lo) || S.state[u] == 2)
                continue;
            if(S.state[u] == 0)
            {
                // first contact: gain = 1 (this edge) - (its other range edges)
                int32_t deg = 0;
                for(int32_t f = G.xadj[u]; f < G.xadj[u + 1]; ++f)
                    deg += (G.adj[f] != u && G.inside(G.adj[f], lo)) ? 1 : 0;
                S.state[u] = 1;
                S.gain[u]  = 2 - deg;  // +1 into left, and the edge no longer counts against
                S.dist[u]  = stamp++;
            }
            else
                S.gain[u] += 2;
            pq.push({S.gain[u], S.dist[u], u});
        }
    };
    take(seed);
    while(taken < want)
    {
        int32_t v = -1;
        while(!pq.empty())
        {
            const Cand c = pq.top();
            pq.pop();
            if(S.state[c.v] == 1 && S.gain[c.v] == c.gain)
            {
                v = c.v;
                break;
            }
        }
        if(v < 0)
        {
            // component used up: the next unreached vertex in range order
            while(scan < hi && S.state[W[scan]] != 0)
                ++scan;
            v = W[scan];
        }
        take(v);
    }
    for(int32_t k = lo; k < hi; ++k)
    {
        S.state[W[k]] = 0;
        S.dist[W[k]]  = -1;
        S.gain[W[k]]  = 0;
    }
}

// cut change when v changes side (positive: the cut shrinks)
int32_t move_gain(const PartGraph& G, int32_t lo, const Scratch& S, int32_t v, int32_t* cross = nullptr)
{
    int32_t same = 0, other = 0;
    for(int32_t e = G.xadj[v]; e < G.xadj[v + 1]; ++e)
    {
        const int32_t u = G.adj[e];
        if(u == v || !G.inside(u, lo))
            continue;
        if(S.side[u] == S.side[v])
            ++same;
        else
            ++other;
    }
    if(cross)
        *cross = other;
    return other - same;
}

bool adjacent(const PartGraph& G, int32_t a, int32_t b)
{
    const int32_t* beg = G.adj + G.xadj[a];
    const int32_t* end = G.adj + G.xadj[a + 1];
    for(const int32_t* p = beg; p != end; ++p)
        if(*p == b)
            return true;
    return false;
}

void refine(const PartGraph& G, int32_t lo, int32_t hi, Scratch& S)
{
    const int32_t* W = G.order.data();
    for(int pass = 0; pass < REFINE_PASSES; ++pass)
    {
        std::priority_queue<Cand> pq[2];
        for(int32_t k = lo; k < hi; ++k)
        {
            const int32_t v     = W[k];
            int32_t       cross = 0;
            const int32_t g     = move_gain(G, lo, S, v, &cross);
            S.gain[v]           = g;
            if(cross > 0)  // boundary vertices; others enter when a neighbour moves
                pq[S.side[v]].push({g, k, v});
        }
        int32_t swaps = 0;
        auto    pop   = [&](int sd) -> int32_t
        {
            while(!pq[sd].empty())
            {
                const Cand c = pq[sd].top();
                pq[sd].pop();
                if(!S.state[c.v] && S.side[c.v] == sd && S.gain[c.v] == c.gain)
                    return c.v;
            }
            return -1;
        };
        for(;;)
        {
            const int32_t a = pop(0), b = pop(1);
            if(a < 0 || b < 0)
                break;
            const int32_t g = S.gain[a] + S.gain[b] - (adjacent(G, a, b) ? 2 : 0);
            if(g <= 0)
                break;
            S.side[a]  = 1;
            S.side[b]  = 0;
            S.state[a] = 1;
            S.state[b] = 1;
            ++swaps;
            for(int32_t x : {a, b})
                for(int32_t e = G.xadj[x]; e < G.xadj[x + 1]; ++e)
                {
                    const int32_t u = G.adj[e];
                    if(u == x || !G.inside(u, lo) || S.state[u])
                        continue;
                    const int32_t gu = move_gain(G, lo, S, u);
                    if(gu != S.gain[u])
                    {
                        S.gain[u] = gu;
                        pq[S.side[u]].push({gu, 0, u});
                    }
                }
        }
        for(int32_t k = lo; k < hi; ++k)
        {
            S.state[W[k]] = 0;
            S.gain[W[k]]  = 0;
        }
        if(swaps == 0)
            break;
    }
}

void bisect_range(PartGraph& G, int32_t lo, int32_t hi, int depth, Scratch& S)
{
    const int32_t m = hi - lo;
    if(m <= G.max_part)
    {
        const int32_t part = lo / G.max_part;
        for(int32_t k = lo; k < hi; ++k)
            G.part_ids[G.order[k]] = part;
        return;
    }
    const int32_t parts_total = (m + G.max_part - 1) / G.max_part;
    int32_t       left        = ((parts_total + 1) / 2) * G.max_part;
    if(left >= m)
        left = m - 1;
    grow_left(G, lo, hi, left, S);
    refine(G, lo, hi, S);
    // left side first, each side in its previous order
    std::stable_partition(G.order.begin() + lo, G.order.begin() + hi, [&](int32_t v) { return S.side[v] == 0; });
    for(int32_t k = lo; k < hi; ++k)
        S.side[G.order[k]] = 0;
    for(int32_t k = lo + left; k < hi; ++k)
        G.tag[G.order[k]].store(lo + left, std::memory_order_relaxed);
    if(depth < PARALLEL_DEPTH && m > 4096)
    {
        auto right = std::async(std::launch::async,
                                [&]
                                {
                                    Scratch own(G.n);
                                    bisect_range(G, lo + left, hi, depth + 1, own);
                                });
        bisect_range(G, lo, lo + left, depth + 1, S);
        right.get();
    }
    else
    {
        bisect_range(G, lo, lo + left, depth + 1, S);
        bisect_range(G, lo + left, hi, depth + 1, S);
    }
}
}  // namespace

void partition_graph(int32_t n, const int32_t* xadj, const int32_t* adj, int32_t max_part, int32_t* part_ids)
{
    PartGraph G{n, xadj, adj, max_part, std::vector<int32_t>(n), std::vector<std::atomic<int32_t>>(n), part_ids};
    for(int32_t v = 0; v < n; ++v)
    {
        G.order[v] = v;
        G.tag[v].store(0, std::memory_order_relaxed);
    }
    Scratch S(n);
    bisect_range(G, 0, n, 0, S);
}
}  // namespace b2s
