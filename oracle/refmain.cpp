// refmain.cpp -- TEST INFRASTRUCTURE: entry wrapper for the reference's own
// driver (cu_test.cu, compiled unchanged with -Dmain=tdfs_ref_main).
//
// cu_test.cu:30 builds its JobQueue through JobQueuePreprocessor, whose
// constructor body is commented out (src/job_queue.h:237-279), so
// JobQueue::q and JobQueue::length are read uninitialised by to_gpu()
// (src/job_queue.h:281-290): with stack garbage that is a cudaMemcpy from a
// wild host pointer.  The kernel only reads JobQueue::cur (initialised to 0),
// so zeroing the stack region the driver's frame will occupy (nvcc compiles
// its host code at -O0: the temporary has its own slot) turns the copy into a
// zero-length no-op without changing the reference's code.
#include <cstring>

int tdfs_ref_main(int argc, char **argv);

__attribute__((noinline)) static void scrub_stack() {
  volatile unsigned char pad[1 << 17];
  std::memset(const_cast<unsigned char *>(pad), 0, sizeof pad);
}

int main(int argc, char **argv) {
  scrub_stack();
  return tdfs_ref_main(argc, argv);
}
