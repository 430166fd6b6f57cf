// ref_detect.cpp -- TEST INFRASTRUCTURE.  Drives the reference's own MTX
// format detection, auto_detect_graph_info (dynamic_update/functions.cpp:35-291,
// compiled from that file, see Makefile), and prints what it detected, so the
// product's detector can be checked against it.
// Usage: ref_detect <file>
// Output: one line "skip header dims weighted laplacian triangle base v_max v_min".
#include <stdio.h>

#include "functions.h"

int main(int argc, char **argv) {
    if (argc < 2) return 2;
    const GraphInfo i = auto_detect_graph_info(argv[1]);
    printf("%ld %d %d %d %d %d %d %ld %ld\n", (long)i.skip_lines, (int)i.has_matrixmarket_header,
           (int)i.has_dimensions_line, (int)i.is_weighted, (int)i.is_laplacian,
           (int)i.is_triangle, i.base, (long)i.v_max, (long)i.v_min);
    return 0;
}
