// ref_readers.cpp -- TEST INFRASTRUCTURE.  Drives the reference's own MTX
// readers (compiled from its functions.cpp, see Makefile) and prints what
// they parsed, so the product's reader can be checked against them:
//   incremental: read_graph (random_walk_incremental/functions.cpp:58-239)
//                read_targets (random_walk_incremental/functions.cpp:261-370)
//   decremental: CSRGraph ctor (random_walk_decremental/functions.cpp:69-281)
//                CSRGraph::read_targets (random_walk_decremental/functions.cpp:303-420)
// Usage: ref_incr_reader graph <file> | targets <file>
//        ref_decr_reader graph <file> | targets <file> <weighted 0|1>
// Output: "V <vert_count>", then "R <v> <deg> <n1> <w1> <n2> <w2> ..." per
// vertex in CSR row order, or "T <count>" then the target array layout.
#include <stdio.h>
#include <string.h>

#include "functions.h"

int main(int argc, char **argv) {
    if (argc < 3) return 2;
#ifdef REF_INCREMENTAL
    if (!strcmp(argv[1], "graph")) {
        CSRGraph g = read_graph(argv[2], true, 0, 1);
#else
    if (!strcmp(argv[1], "graph")) {
        CSRGraph g(argv[2], true, 0, 1);
#endif
        printf("V %zu\n", (size_t)g.vert_count);
        for (size_t v = 0; v < g.vert_count; ++v) {
            printf("R %zu %u", v, (unsigned)(g.begin[v + 1] - g.begin[v]));
            for (size_t j = g.begin[v]; j < g.begin[v + 1]; ++j)
                printf(" %u %.9g", (unsigned)g.adj[j], (double)g.weight[j]);
            printf("\n");
        }
        return 0;
    }
    if (!strcmp(argv[1], "targets")) {
#ifdef REF_INCREMENTAL
        Targets t = read_targets(argv[2], -1, 1);
        printf("T %zu\n", t.target_count);
        for (size_t i = 0; i < 2 * t.target_count; ++i) printf("N %u\n", (unsigned)t.nodes[i]);
        for (size_t i = 0; i < t.target_count; ++i) printf("W %.9g\n", (double)t.weights[i]);
        t.nodes = new vertex_t[1];
        t.weights = new weight_t[1];
#else
        int weighted = argc > 3 ? atoi(argv[3]) : 0;
        CSRGraph g;
        g.read_targets(argv[2], -1, weighted, 10);
        printf("T %zu\n", (size_t)g.sample_count);
        for (size_t i = 0; i < 2 * g.sample_count; ++i) printf("N %u\n", (unsigned)g.sample_nodes[i]);
#endif
        return 0;
    }
    return 2;
}
