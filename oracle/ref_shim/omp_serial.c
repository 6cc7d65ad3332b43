/* Test infrastructure: the one OpenMP runtime call of the reference's
 * avx512 kernel (LinearBasis/avx512/src/InterpolateArray.cpp), answered for a
 * build without -fopenmp, where its parallel regions run on one thread. */
int omp_get_thread_num(void) { return 0; }
