// ref_serial_stub.cpp -- TEST INFRASTRUCTURE ONLY. The reference's finite-volume operators (fvc.cu) end a
// halo exchange with Pstream::waitAll, whose definition (src/parallel/pstream/cf_pstream.cu) needs MPI,
// which this image lacks. The shim drives one serial process with no processor patches, so nothing is
// ever pending: completing no requests is what waitAll does there. Bound inside libref.so only.
#include "cf_pstream.cuh"

void brae::Pstream::waitAll() {}
