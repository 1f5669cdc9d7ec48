// One-thread stand-in for the OpenMP runtime calls of the reference's
// training program (Training.cpp sets the thread count around its updates),
// written for this project and used ONLY to build the reference's nnp-train
// into the test oracle; its parallel pragmas are compiled without OpenMP.
#ifndef N2P2B200_OMP_STUB_H
#define N2P2B200_OMP_STUB_H

inline int omp_get_max_threads() { return 1; }
inline int omp_get_num_threads() { return 1; }
inline int omp_get_thread_num() { return 0; }
inline void omp_set_num_threads(int) {}

#endif
