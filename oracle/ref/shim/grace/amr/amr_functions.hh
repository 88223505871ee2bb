// Stand-in for GRACE's AMR forest helpers: the ghost-zone index helpers
// include it only for the p4est element counts of a 3-D forest.
#pragma once
#ifndef P4EST_FACES
#define P4EST_FACES 6
#endif
#ifndef P4EST_CHILDREN
#define P4EST_CHILDREN 8
#endif
#ifndef P8EST_EDGES
#define P8EST_EDGES 12
#endif
