/* ref_blk_compat.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Included ahead of the reference's eigen/src/lanczos_blk.c by
 * oracle/build_ref.sh (g++ -include), which compiles that file with the
 * reference's NoGnuStatementExpre switch: Allreduce_MPI_sp is then a
 * function, declared by the reference for double pointers.  lanczos_blk.c
 * also passes complex pointers with MPI's count of doubles
 * (dot_product, lanczos_blk.c:172; mult_dot_product_hermitian, 215), so this
 * adds that overload; both are defined in oracle/ref_lanczos_driver.cc with
 * MPI's meaning on one rank: copy `count` doubles.  (The serial build's
 * default macro copies `count` elements of the pointer's type, 32 bytes
 * into dot_product's caller's 16-byte result.) */
#ifndef REF_BLK_COMPAT_H
#define REF_BLK_COMPAT_H
#include <cstring>
#include "nml_dcscalar.h"
#include "mpi_fake.h"
void Allreduce_MPI_sp(nml_dcomplex *pa, nml_dcomplex *pb, int count, MPI_Datatype datatype,
                      MPI_Op op, MPI_Comm comm);
#endif
