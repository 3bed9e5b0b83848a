/* A plain MPI application, linked `-ltempi_b200 -lminimpi`: MPI_Pack and
   MPI_Type_commit resolve to the interposer, which reaches the library's
   definitions through dlsym(RTLD_NEXT).  Packs the 1024 x 64 B vector
   (stride 512 B) from host memory and checks every byte. */
#include <mpi.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "tempi_b200.h"

int main(int argc, char **argv) {
  if (MPI_Init(&argc, &argv) != MPI_SUCCESS) return 1;
  MPI_Datatype t;
  MPI_Type_vector(1024, 64, 512, MPI_BYTE, &t);
  if (MPI_Type_commit(&t) != MPI_SUCCESS) return 2;
  tempi_desc d;
  if (tempi_describe(t, &d) != TEMPI_OK || d.block != 64 || d.counts[0] != 1024)
    return 3;
  unsigned char *src = malloc(524288), *out = malloc(65536);
  for (int i = 0; i < 524288; ++i) src[i] = (unsigned char)(i * 7 + 3);
  int pos = 0;
  if (MPI_Pack(src, 1, t, out, 65536, &pos, MPI_COMM_WORLD) != MPI_SUCCESS || pos != 65536)
    return 4;
  for (int r = 0; r < 1024; ++r)
    if (memcmp(out + 64 * r, src + 512 * r, 64)) return 5;
  pos = 0;
  if (MPI_Pack(src, 1, t, out, 100, &pos, MPI_COMM_WORLD) != MPI_ERR_TRUNCATE) return 6;
  MPI_Type_free(&t);
  MPI_Finalize();
  printf("OK\n");
  return 0;
}
