// Column-major multi-index helpers with escript's INDEXn names (first index fastest).
#pragma once
#define INDEX2(i, j, N0) ((i) + (N0) * (j))
#define INDEX3(i, j, k, N0, N1) ((i) + (N0) * INDEX2(j, k, N1))
#define INDEX4(i, j, k, l, N0, N1, N2) ((i) + (N0) * INDEX3(j, k, l, N1, N2))
#define INDEX5(i, j, k, l, m, N0, N1, N2, N3) ((i) + (N0) * INDEX4(j, k, l, m, N1, N2, N3))
