// me_driver.cpp -- the inversion driver: what the reference's MEINV program
// does around INVERSION_MULTI (Src/ME_INV.c:64-295, Src/IO.c:120-742,
// Src/INV_INIT.c:207-250), on one or several GPUs.
//
//   * reads the Stokes cube [nw][4][nx][ny] (BITPIX 16 / -32 / -64) and the
//     wavelength grid from FITS (rWavelength, rProfile, rProfilesll);
//   * inverts the pixels of sol_box in raster order in chunks of `nprofiles`
//     (INIT_INV's nProf; one chunk of all of them with Cache_prof);
//   * writes res.fits [10][nx'][ny'] and, with output_fit, fit.fits
//     [nw][4][nx'][ny'] (CACHE_INIT, WRITE_RESULT);
//   * with Cache_inv, keeps the reference's checkpoint file (16-byte header
//     "cach", nx', ny', ncache, then one int per chunk set to 1 once the chunk
//     is written) and skips the chunks it marks done (PixelMV).
//
// GPU batching: consecutive chunks that still need work are inverted
// together, up to `batch_pixels` per call; each chunk's results and cache flag
// are written as the reference writes them, so the files are the same.  With
// several GPUs, batch b goes to plan b mod N (the reference farms chunks to
// MPI workers first-come; a static assignment keeps runs reproducible).  Each
// plan carries the LM chi^2 from pixel to pixel over its own batches, as each
// reference process does over its own chunks.
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/me_b200.h"

namespace me {
int record_error(int code, const char *msg);
}

namespace {

int fail(int code, const std::string &m) { return me::record_error(code, m.c_str()); }

struct CacheHeader {  // the reference's packed STRUCT_CACHE (Src/RINPUT.h:97-104)
  char magic[4];
  int32_t nx, ny, ncache;
};
static_assert(sizeof(CacheHeader) == 16, "cache header is 16 bytes");

struct Job {
  long first_chunk, nchunks;  // chunks [first_chunk, first_chunk + nchunks)
  long first_pixel, npix;     // raster pixels of sol_box
};

}  // namespace

extern "C" int me_run_options_default(me_run_options *o) {
  if (!o) return fail(ME_ERR_ARG, "null argument");
  memset(o, 0, sizeof(*o));
  o->ndevices = 1;
  o->batch_pixels = 131072;
  o->max_group = -1;
  o->tail_slots = -2;
  return ME_OK;
}

extern "C" int me_run_config(const me_config *cfg, const me_run_options *opt_in,
                             me_run_report *rep) {
  if (!cfg) return fail(ME_ERR_ARG, "null config");
  me_run_options opt;
  if (opt_in)
    opt = *opt_in;
  else
    me_run_options_default(&opt);
  if (opt.ndevices < 1) opt.ndevices = 1;
  if (opt.batch_pixels < 1) opt.batch_pixels = 131072;
  const auto t0 = std::chrono::steady_clock::now();
  me_run_report r;
  memset(&r, 0, sizeof r);

  // ---- the data cube and the wavelengths (rWavelength) ----
  int bitpix = 0, naxis = 0;
  long naxes[8];
  int rc = me_fits_image_info(cfg->data_path, &bitpix, &naxis, naxes);
  if (rc) return rc;
  if (naxis < 3 || naxis > 4) return fail(ME_ERR_FORMAT, "wrong dimension of the data hdu");
  if (naxes[1] != 4) return fail(ME_ERR_FORMAT, "wrong size of the data hdu");
  if (bitpix != 16 && bitpix != -32 && bitpix != -64)
    return fail(ME_ERR_FORMAT, "error in the data type of data hdu: bitpix = " +
                                   std::to_string(bitpix));
  const long nw = naxes[0], nx = naxes[2], ny = naxis == 4 ? naxes[3] : 1;
  int wb = 0, wn = 0;
  long wx[8];
  rc = me_fits_image_info(cfg->wavelength_path, &wb, &wn, wx);
  if (rc) return rc;
  if (wn != 1) return fail(ME_ERR_FORMAT, "error in the dimension of wavelength hdu");
  if (wx[0] != nw) return fail(ME_ERR_FORMAT, "wavelength is not consistent with the profile");
  if (wb != -32 && wb != -64) return fail(ME_ERR_FORMAT, "error in the data type of the wavelength hdu");
  if (nw > ME_MAX_NL) return fail(ME_ERR_FORMAT, "wavelength grid larger than ME_MAX_NL");
  std::vector<double> lambda(nw);
  rc = me_fits_read(cfg->wavelength_path, 0, nw, lambda.data());
  if (rc) return rc;

  // ---- sol_box (rWavelength's checks) and the chunks (INIT_INV) ----
  long x0 = cfg->sol_box[0], x1 = cfg->sol_box[1], y0 = cfg->sol_box[2], y1 = cfg->sol_box[3];
  if (x0 < 0 || x0 >= nx) x0 = 0;
  if (x1 < 0 || x1 >= nx) x1 = nx - 1;
  if (y0 < 0 || y0 >= ny) y0 = 0;
  if (y1 < 0 || y1 >= ny) y1 = ny - 1;
  if (x1 < x0 || y1 < y0) return fail(ME_ERR_CONFIG, "sol_box is empty");
  const long nxc = x1 - x0 + 1, nyc = y1 - y0 + 1, counts = nxc * nyc;
  long nprof = cfg->nprofiles;
  if (nprof < 1) nprof = 1;
  if (nprof > counts) nprof = counts;
  if (cfg->cache_prof) nprof = counts;
  const long ncache = counts / nprof + 1;
  const long nchunks = (counts + nprof - 1) / nprof;
  const bool use_cache = cfg->cache_inv && !cfg->cache_prof;
  const bool want_fit = cfg->output_fit && !cfg->cache_prof;
  r.nx = nx;
  r.ny = ny;
  r.nw = nw;
  r.counts = counts;
  r.chunk_pixels = nprof;
  r.nchunks = nchunks;

  // ---- the checkpoint and the output files (CACHE_INIT) ----
  std::vector<int32_t> done(ncache, 0);
  bool resume = false;
  if (use_cache) {
    FILE *f = fopen(cfg->cache_path, "rb");
    if (f) {
      CacheHeader h;
      if (fread(&h, sizeof h, 1, f) == 1 && memcmp(h.magic, "cach", 4) == 0 && h.nx == nxc &&
          h.ny == nyc && h.ncache == ncache &&
          fread(done.data(), sizeof(int32_t), (size_t)ncache, f) == (size_t)ncache)
        resume = true;
      else
        std::fill(done.begin(), done.end(), 0);
      fclose(f);
    }
  }
  if (resume) {
    int b2, n2;
    long a2[8];
    rc = me_fits_image_info(cfg->result_path, &b2, &n2, a2);
    if (rc) return rc;
    if (n2 != 3 || a2[0] != 10 || a2[1] != nxc || a2[2] != nyc || b2 != -64)
      return fail(ME_ERR_FORMAT, "wrong size of the result file");
    if (want_fit) {
      rc = me_fits_image_info(cfg->fit_path, &b2, &n2, a2);
      if (rc) return rc;
      if (n2 != 4 || a2[0] != nw || a2[1] != 4 || a2[2] != nxc || a2[3] != nyc || b2 != -64)
        return fail(ME_ERR_FORMAT, "wrong size of the fit file");
    }
  } else {
    if (use_cache) {
      FILE *f = fopen(cfg->cache_path, "wb");
      if (!f) return fail(ME_ERR_IO, std::string("cannot create ") + cfg->cache_path);
      CacheHeader h;
      memcpy(h.magic, "cach", 4);
      h.nx = (int32_t)nxc;
      h.ny = (int32_t)nyc;
      h.ncache = (int32_t)ncache;
      bool ok = fwrite(&h, sizeof h, 1, f) == 1 &&
                fwrite(done.data(), sizeof(int32_t), (size_t)ncache, f) == (size_t)ncache;
      ok = (fclose(f) == 0) && ok;
      if (!ok) return fail(ME_ERR_IO, std::string("cannot write ") + cfg->cache_path);
    }
    const long rdim[3] = {10, nxc, nyc};
    rc = me_fits_create(cfg->result_path, 3, rdim);
    if (rc) return rc;
    if (want_fit) {
      const long fdim[4] = {nw, 4, nxc, nyc};
      rc = me_fits_create(cfg->fit_path, 4, fdim);
      if (rc) return rc;
    }
  }

  // ---- the work: runs of chunks still to do, cut into batches ----
  std::vector<Job> jobs;
  long budget = opt.stop_after_chunks > 0 ? opt.stop_after_chunks : nchunks;
  const long per_batch = std::max(1L, opt.batch_pixels / nprof);
  for (long c = 0; c < nchunks && budget > 0;) {
    if (done[c]) {
      r.chunks_skipped++;
      c++;
      continue;
    }
    long e = c;
    while (e < nchunks && !done[e] && e - c < per_batch && e - c < budget) e++;
    Job j;
    j.first_chunk = c;
    j.nchunks = e - c;
    j.first_pixel = c * nprof;
    j.npix = std::min(counts, e * nprof) - j.first_pixel;
    jobs.push_back(j);
    budget -= e - c;
    c = e;
  }

  // ---- one plan per device, batches b, b + N, ... on plan b mod N ----
  const int nd = opt.ndevices;
  std::vector<me_plan *> plans(nd, nullptr);
  for (int d = 0; d < nd; d++) {
    const int dev = opt.devices ? opt.devices[d] : d;
    rc = me_plan_create(cfg, lambda.data(), (int)nw, dev, &plans[d]);
    if (!rc && opt.max_group >= 0) me_plan_set_max_group(plans[d], opt.max_group);
    if (!rc && opt.tail_slots >= -1) me_plan_set_tail_slots(plans[d], opt.tail_slots);
    if (!rc && opt.initializer) rc = me_plan_set_initializer(plans[d], opt.initializer);
    if (rc) {
      for (me_plan *p : plans)
        if (p) me_plan_destroy(p);
      return rc;
    }
  }
  std::mutex io;  // file writes and the error slot
  int first_rc = ME_OK;
  std::string first_msg;
  std::atomic<long> pixels(0), chunks_done(0);
  auto worker = [&](int d) {
    std::vector<double> prof, res, fit;
    for (size_t b = (size_t)d; b < jobs.size(); b += (size_t)nd) {
      {
        std::lock_guard<std::mutex> g(io);
        if (first_rc) return;
      }
      const Job &j = jobs[b];
      prof.resize((size_t)j.npix * 4 * nw);
      res.resize((size_t)j.npix * 10);
      if (want_fit) fit.resize((size_t)j.npix * 4 * nw);
      // profiles of raster pixels [first, first + n): row segments of sol_box
      int e = ME_OK;
      for (long k = 0; k < j.npix && !e;) {
        const long idx = j.first_pixel + k;
        const long yy = y0 + idx / nxc, xx = x0 + idx % nxc;
        const long run = std::min(j.npix - k, x1 - xx + 1);
        e = me_fits_read(cfg->data_path, (yy * nx + xx) * 4 * nw, run * 4 * nw,
                         prof.data() + (size_t)k * 4 * nw);
        k += run;
      }
      if (!e)
        e = me_invert_batch(plans[d], prof.data(), j.npix, res.data(),
                            want_fit ? fit.data() : nullptr, nullptr);
      std::lock_guard<std::mutex> g(io);
      if (!e) e = me_fits_write(cfg->result_path, j.first_pixel * 10, j.npix * 10, res.data());
      if (!e && want_fit)
        e = me_fits_write(cfg->fit_path, j.first_pixel * 4 * nw, j.npix * 4 * nw, fit.data());
      if (!e && use_cache) {
        FILE *f = fopen(cfg->cache_path, "r+b");
        if (!f) {
          e = fail(ME_ERR_IO, std::string("cannot update ") + cfg->cache_path);
        } else {
          const int32_t one = 1;
          for (long c = j.first_chunk; c < j.first_chunk + j.nchunks && !e; c++)
            if (fseek(f, (long)sizeof(CacheHeader) + c * 4, SEEK_SET) != 0 ||
                fwrite(&one, 4, 1, f) != 1)
              e = fail(ME_ERR_IO, std::string("cannot update ") + cfg->cache_path);
          if (fclose(f) != 0 && !e) e = fail(ME_ERR_IO, std::string("cannot update ") + cfg->cache_path);
        }
      }
      if (e) {
        if (!first_rc) {
          first_rc = e;
          first_msg = me_last_error();
        }
        return;
      }
      pixels += j.npix;
      chunks_done += j.nchunks;
    }
  };
  std::vector<std::thread> threads;
  for (int d = 1; d < nd; d++) threads.emplace_back(worker, d);
  worker(0);
  for (auto &t : threads) t.join();
  for (me_plan *p : plans) me_plan_destroy(p);
  if (first_rc) return fail(first_rc, first_msg);
  r.chunks_done = chunks_done;
  r.pixels_inverted = pixels;
  r.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (rep) *rep = r;
  return ME_OK;
}

extern "C" int me_run(const char *ctl_path, const me_run_options *opt, me_run_report *rep) {
  if (!ctl_path) return fail(ME_ERR_ARG, "null path");
  me_config cfg;
  char err[512];
  const int rc = me_config_parse(ctl_path, &cfg, err, sizeof err);
  if (rc) return fail(rc, err);
  return me_run_config(&cfg, opt, rep);
}
