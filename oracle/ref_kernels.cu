// ORACLE -- test infrastructure only.  Never linked into the product.
//
// Thin extern "C" driver around the reference's own packer kernels, compiled
// straight from the reference sources (include/pack_kernels.cuh and the
// headers it includes) by oracle/build_ref.sh into oracle/_ref/.  It launches
// them exactly as the reference does:
//   2-D: Pack2DConfig (pack_kernels.cuh:122-175) and the launch in
//        Packer2D::launch_pack/unpack (src/internal/packer_2d.cu:21-74);
//   3-D: the word-size and grid rules of the Packer3D constructor
//        (src/internal/packer_3d.cu:19-78, restated here because that file
//        pulls in the MPI-dependent logging headers) and the launch in
//        launch_pack/unpack (:80-115).
// Used by the GPU tests as "the reference TEMPI packer output" and timed
// there as the reference-kernel baseline.
#include "pack_kernels.cuh"

#include <algorithm>
#include <cstdint>

namespace {
using Fn3 = void (*)(void *__restrict__, const void *__restrict__, const int,
                     unsigned, unsigned, unsigned, unsigned, unsigned,
                     uint64_t);

int word3(unsigned off, unsigned bl) {
  if (bl % 12 == 0 && off % 12 == 0) return 4;
  if (bl % 8 == 0 && off % 8 == 0) return 8;
  if (bl % 6 == 0 && off % 6 == 0) return 6;
  if (bl % 4 == 0 && off % 4 == 0) return 4;
  if (bl % 3 == 0 && off % 3 == 0) return 3;
  if (bl % 2 == 0 && off % 2 == 0) return 2;
  return 1;
}

template <bool UNPACK> Fn3 fn3(int w) {
  switch (w) {
  case 8: return UNPACK ? static_cast<Fn3>(unpack_3d<8>) : static_cast<Fn3>(pack_3d<8>);
  case 6: return UNPACK ? static_cast<Fn3>(unpack_3d<6>) : static_cast<Fn3>(pack_3d<6>);
  case 4: return UNPACK ? static_cast<Fn3>(unpack_3d<4>) : static_cast<Fn3>(pack_3d<4>);
  case 3: return UNPACK ? static_cast<Fn3>(unpack_3d<3>) : static_cast<Fn3>(pack_3d<3>);
  case 2: return UNPACK ? static_cast<Fn3>(unpack_3d<2>) : static_cast<Fn3>(pack_3d<2>);
  default: return UNPACK ? static_cast<Fn3>(unpack_3d<1>) : static_cast<Fn3>(pack_3d<1>);
  }
}
} // namespace

// typed = object origin (the reference adds the start offset itself)
extern "C" int ref_pack_2d(int unpack, void *typed, void *packed, int incount,
                           unsigned off, unsigned bl, unsigned count,
                           unsigned stride, unsigned extent, void *stream) {
  Pack2DConfig cfg(off, bl, count);
  char *t = static_cast<char *>(typed) + off;
  if (unpack)
    cfg.unpackfn<<<cfg.dim_grid(incount), cfg.dim_block(), 0,
                   (cudaStream_t)stream>>>(t, packed, incount, bl, count,
                                           stride, extent);
  else
    cfg.packfn<<<cfg.dim_grid(incount), cfg.dim_block(), 0,
                 (cudaStream_t)stream>>>(packed, t, incount, bl, count, stride,
                                         extent);
  return (int)cudaGetLastError();
}

extern "C" int ref_pack_3d(int unpack, void *typed, void *packed, int incount,
                           unsigned off, unsigned bl, unsigned c1, unsigned s1,
                           unsigned c2, unsigned s2, unsigned extent,
                           void *stream) {
  const int w = word3(off, bl);
  Dim3 bd = Dim3::fill_xyz_by_pow2(Dim3(bl / w, c1, c2), 512);
  Dim3 gd = (Dim3(bl / w, c1, c2) + bd - Dim3(1, 1, 1)) / bd;
  gd.y = std::min(int64_t(65535), gd.y);
  char *t = static_cast<char *>(typed) + off;
  if (unpack)
    fn3<true>(w)<<<gd, bd, 0, (cudaStream_t)stream>>>(t, packed, incount, bl,
                                                       c1, s1, c2, s2, extent);
  else
    fn3<false>(w)<<<gd, bd, 0, (cudaStream_t)stream>>>(packed, t, incount, bl,
                                                        c1, s1, c2, s2, extent);
  return (int)cudaGetLastError();
}
