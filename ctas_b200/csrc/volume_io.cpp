// volume_io.cpp -- raw contiguous volumes for the streamed volume call
// (ctas_vol_raw_reconstruct, include/ctas_volume.h).
//
// The reference's fast path for large volumes memory-maps a contiguous,
// unfiltered float32 HDF5 dataset (or any file under /dev/shm or a
// CTAS_MMAP_PATH prefix) and reads / writes slices straight from / into the
// mapping (HDFwrapper::mmapMeIfYouCan, src/common/external.world.cpp:
// 191-280).  This file serves the same layout -- a [slices][rows][cols] array
// at a byte offset of a file -- with positioned reads and writes, split over
// a few threads per chunk so that a page-cache or tmpfs file moves at memory
// speed into the pinned ring of the volume call.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ctas_volume.h"
#include "fbp_host.hpp"

namespace {

template <class F> int guarded(F &&f) {
  try {
    return f();
  } catch (const ctas::Error &e) {
    ctas::set_last_error(e.msg);
    return e.code;
  } catch (const std::bad_alloc &) {
    ctas::set_last_error("host allocation failed");
    return CTAS_E_NOMEM;
  } catch (const std::exception &e) {
    ctas::set_last_error(e.what());
    return CTAS_E_ARG;
  }
}

// One positioned transfer of `bytes` at file offset `off`, resumed after
// short transfers; returns 0 or an errno value (EIO for an early end of file).
int transfer(bool write, int fd, char *buf, size_t bytes, off_t off) {
  while (bytes > 0) {
    const ssize_t n = write ? ::pwrite(fd, buf, bytes, off) : ::pread(fd, buf, bytes, off);
    if (n < 0) {
      if (errno == EINTR) continue;
      return errno;
    }
    if (n == 0) return EIO;
    buf += n;
    bytes -= (size_t)n;
    off += n;
  }
  return 0;
}

// The transfer split into `threads` contiguous parts of whole MiB.
int par_transfer(bool write, int fd, char *buf, size_t bytes, off_t off, int threads) {
  const size_t mib = size_t(1) << 20;
  const size_t per = std::max(mib, (bytes / (size_t)std::max(1, threads) + mib - 1) / mib * mib);
  const int parts = (int)((bytes + per - 1) / per);
  if (parts <= 1) return transfer(write, fd, buf, bytes, off);
  std::vector<int> rc((size_t)parts, 0);
  std::vector<std::thread> th;
  th.reserve((size_t)parts - 1);
  for (int i = 1; i < parts; i++) {
    const size_t a = per * (size_t)i, n = std::min(per, bytes - a);
    th.emplace_back([=, &rc] { rc[(size_t)i] = transfer(write, fd, buf + a, n, off + (off_t)a); });
  }
  rc[0] = transfer(write, fd, buf, std::min(per, bytes), off);
  for (auto &t : th) t.join();
  for (int r : rc)
    if (r) return r;
  return 0;
}

struct RawIO {
  int fd_in = -1, fd_out = -1;
  int64_t in_off = 0, out_off = 0, in_slice = 0, out_slice = 0;
  int threads = 1;
  int err = 0;  // errno of the first failure
  ~RawIO() {
    if (fd_in >= 0) ::close(fd_in);
    if (fd_out >= 0) ::close(fd_out);
  }
};

int raw_read(void *user, int64_t first, int64_t count, float *sinos) {
  auto *io = static_cast<RawIO *>(user);
  const int r = par_transfer(false, io->fd_in, reinterpret_cast<char *>(sinos),
                             (size_t)(count * io->in_slice),
                             (off_t)(io->in_off + first * io->in_slice), io->threads);
  if (r && !io->err) io->err = r;
  return r;
}

int raw_write(void *user, int64_t first, int64_t count, const void *slices) {
  auto *io = static_cast<RawIO *>(user);
  const int r = par_transfer(true, io->fd_out,
                             const_cast<char *>(static_cast<const char *>(slices)),
                             (size_t)(count * io->out_slice),
                             (off_t)(io->out_off + first * io->out_slice), io->threads);
  if (r && !io->err) io->err = r;
  return r;
}

}  // namespace

extern "C" {

int ctas_vol_raw_reconstruct(ctas_fbp *h, const char *in_path, int64_t in_offset,
                             int64_t n_slices, const char *out_path, int64_t out_offset,
                             float center, int32_t bpp, float mincon, float maxcon,
                             int32_t io_threads) {
  return guarded([&] {
    if (!h || !in_path || !out_path) ctas::fail(CTAS_E_ARG, "null argument");
    if (in_offset < 0 || out_offset < 0 || n_slices < 0 || io_threads < 0)
      ctas::fail(CTAS_E_ARG, "negative offset, slice count or thread count");
    const int32_t sb = ctas_vol_sample_bytes(bpp);
    if (sb == 0) ctas::fail(CTAS_E_ARG, "bits per sample must be 0, +-8, +-16, +-32 or +-64");
    int64_t N = 0, W = 0, rows = 0, cols = 0;
    int rc = ctas_fbp_sino_shape(h, &N, &W);
    if (rc == CTAS_OK) rc = ctas_fbp_out_shape(h, &rows, &cols);
    if (rc != CTAS_OK) return rc;
    RawIO io;
    io.in_off = in_offset;
    io.out_off = out_offset;
    io.in_slice = (int64_t)sizeof(float) * N * W;
    io.out_slice = (int64_t)sb * rows * cols;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    io.threads = io_threads > 0 ? io_threads : (int)std::min(8u, std::max(1u, hw / 4));
    io.fd_in = ::open(in_path, O_RDONLY | O_CLOEXEC);
    if (io.fd_in < 0)
      ctas::fail(CTAS_E_IO, std::string("cannot open ") + in_path + ": " + std::strerror(errno));
    struct stat st {};
    if (::fstat(io.fd_in, &st) != 0)
      ctas::fail(CTAS_E_IO, std::string("cannot stat ") + in_path + ": " + std::strerror(errno));
    if ((int64_t)st.st_size < in_offset + n_slices * io.in_slice)
      ctas::fail(CTAS_E_IO, std::string(in_path) + " holds " + std::to_string(st.st_size) +
                                " bytes; " + std::to_string(n_slices) + " sinograms of " +
                                std::to_string(N) + " x " + std::to_string(W) +
                                " float32 at offset " + std::to_string(in_offset) + " need " +
                                std::to_string(in_offset + n_slices * io.in_slice));
#ifdef POSIX_FADV_SEQUENTIAL
    ::posix_fadvise(io.fd_in, (off_t)in_offset, (off_t)(n_slices * io.in_slice),
                    POSIX_FADV_SEQUENTIAL);
#endif
    io.fd_out = ::open(out_path, O_WRONLY | O_CREAT | O_CLOEXEC, 0644);
    if (io.fd_out < 0)
      ctas::fail(CTAS_E_IO, std::string("cannot open ") + out_path + ": " + std::strerror(errno));
    rc = ctas_fbp_reconstruct_volume(h, n_slices, center, bpp, mincon, maxcon, raw_read,
                                     raw_write, &io);
    if (rc == CTAS_E_IO && io.err)
      ctas::fail(CTAS_E_IO, std::string(ctas_fbp_last_error()) + " (" + std::strerror(io.err) + ")");
    return rc;
  });
}

}  // extern "C"
