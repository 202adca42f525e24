// gadget2.cu -- Gadget-2 files of particle data: the lightcone output and
// snapshots.
//
// Layout (the reference's serial writer, Particles_gevolution.hpp:826-840, and
// its MPI-IO twin :300-323): four blocks, each enclosed by a uint32 record
// length before and after it --
//   header   256 bytes (gadget2_header, metadata.hpp:159-178)
//   POS      3 n float    (kpc/h: box units times hdr.BoxSize)
//   VEL      3 n float    (Gadget velocity units)
//   ID       n int64      (GADGET_ID_BYTES = 8)
// The writer sets npart[1], npartTotal[1] and npartTotalHW[1] from n, as the
// reference does for its single particle species; the other header fields are
// the caller's (output.hpp:2097-2123 shows how the reference fills them).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "gev.h"

static_assert(sizeof(gev_gadget2_header) == 256, "Gadget-2 header must be 256 bytes");

namespace {

bool write_block(FILE *f, const void *data, uint64_t bytes)
{
    const uint32_t len = (uint32_t)bytes;   // the format's record length is 32-bit, like the reference's
    return fwrite(&len, 4, 1, f) == 1 && (bytes == 0 || fwrite(data, 1, bytes, f) == bytes) && fwrite(&len, 4, 1, f) == 1;
}

int write_file(const char *path, const gev_gadget2_header *hdr_in, const float *pos, const float *vel, const int64_t *ids,
               int64_t n)
{
    gev_gadget2_header hdr = *hdr_in;
    hdr.npart[1] = (uint32_t)n;
    hdr.npartTotal[1] = (uint32_t)((uint64_t)n & 0xffffffffull);
    hdr.npartTotalHW[1] = (uint32_t)((uint64_t)n >> 32);
    FILE *f = fopen(path, "wb");
    if (!f) return GEV_ERR_ARG;
    bool ok = write_block(f, &hdr, sizeof hdr) && write_block(f, pos, (uint64_t)n * 3 * sizeof(float)) &&
              write_block(f, vel, (uint64_t)n * 3 * sizeof(float)) && write_block(f, ids, (uint64_t)n * sizeof(int64_t));
    ok = (fclose(f) == 0) && ok;
    return ok ? GEV_OK : GEV_ERR_ARG;
}

// one record: its leading length must be `bytes`, and so must its trailing one
bool read_block(FILE *f, void *data, uint64_t bytes)
{
    uint32_t len0 = 0, len1 = 0;
    if (fread(&len0, 4, 1, f) != 1 || len0 != (uint32_t)bytes) return false;
    if (bytes > 0 && fread(data, 1, bytes, f) != bytes) return false;
    return fread(&len1, 4, 1, f) == 1 && len1 == len0;
}

// the header, then the particle count of species 1 (npartTotal[1] + 2^32 npartTotalHW[1])
int read_header(FILE *f, gev_gadget2_header *hdr, int64_t *n)
{
    if (!read_block(f, hdr, sizeof *hdr)) return GEV_ERR_ARG;
    const uint64_t total = (uint64_t)hdr->npartTotal[1] + ((uint64_t)hdr->npartTotalHW[1] << 32);
    // one file of a set holds npart[1] particles; a single file holds them all
    *n = (int64_t)(hdr->num_files > 1 ? (uint64_t)hdr->npart[1] : total);
    for (int s = 0; s < 6; s++)
        if (s != 1 && hdr->npart[s] != 0) return GEV_ERR_ARG;   // one particle species (CDM), as the writers here
    return GEV_OK;
}

}  // namespace

extern "C" {

int gev_gadget2_read(const char *path, gev_gadget2_header *hdr, float *pos, float *vel, int64_t *ids, int64_t capacity,
                     int64_t *n_out)
{
    if (!path || !hdr || !n_out || capacity < 0) return GEV_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return GEV_ERR_ARG;
    int64_t n = 0;
    int rc = read_header(f, hdr, &n);
    if (rc == GEV_OK) {
        *n_out = n;
        if (!pos && !vel && !ids) {
            fclose(f);
            return GEV_OK;   // header and count only
        }
        if (n > capacity || (n > 0 && (!pos || !vel || !ids))) rc = GEV_ERR_CAPACITY;
        else if (!read_block(f, pos, (uint64_t)n * 3 * sizeof(float)) || !read_block(f, vel, (uint64_t)n * 3 * sizeof(float)) ||
                 !read_block(f, ids, (uint64_t)n * sizeof(int64_t)))
            rc = GEV_ERR_ARG;
    }
    fclose(f);
    return rc;
}

int gev_gadget2_write(const char *path, const gev_gadget2_header *hdr, const float *pos, const float *vel,
                      const int64_t *ids, int64_t n)
{
    if (!path || !hdr || n < 0 || (n > 0 && (!pos || !vel || !ids))) return GEV_ERR_ARG;
    if ((uint64_t)n * 3 * sizeof(float) > 0xffffffffull) return GEV_ERR_ARG;   // record length does not fit 32 bits
    return write_file(path, hdr, pos, vel, ids, n);
}

int gev_particles_load_gadget2(gev_ctx *ctx, const char *path, double mass, gev_gadget2_header *hdr_out)
{
    if (!ctx || !path) return GEV_ERR_ARG;
    gev_gadget2_header hdr;
    int64_t n = 0;
    int rc = gev_gadget2_read(path, &hdr, nullptr, nullptr, nullptr, 0, &n);
    if (rc != GEV_OK) return rc;
    if (hdr.time <= 0.0 || hdr.BoxSize <= 0.0) return GEV_ERR_ARG;
    std::vector<float> pos(3 * (size_t)n), vel(3 * (size_t)n);
    std::vector<int64_t> ids((size_t)n);
    rc = gev_gadget2_read(path, &hdr, pos.data(), vel.data(), ids.data(), n, &n);
    if (rc != GEV_OK) return rc;
    // perfParticles_gevolution::loadGadget2 (Particles_gevolution.hpp:2565-2568):
    // box units = pos / BoxSize, momentum = vel * a / (1 / sqrt(a) / GADGET_VELOCITY_CONVERSION)
    const double rescale_vel = 1.0 / 3.335640952e-6 / std::sqrt(hdr.time);
    std::vector<double> p(3 * (size_t)n), q(3 * (size_t)n);
    for (size_t i = 0; i < 3 * (size_t)n; i++) {
        p[i] = (double)pos[i] / hdr.BoxSize;
        q[i] = (double)vel[i] * hdr.time / rescale_vel;
    }
    rc = gev_particles_set(ctx, p.data(), q.data(), ids.data(), n, mass);
    if (rc == GEV_OK && hdr_out) *hdr_out = hdr;
    return rc;
}

int gev_snapshot_gadget2(gev_ctx *ctx, const char *path, const gev_gadget2_header *hdr, int32_t tracer_factor)
{
    if (!ctx || !path || !hdr || tracer_factor < 1 || hdr->time <= 0.0) return GEV_ERR_ARG;
    int64_t n = 0;
    int rc = gev_particles_count(ctx, &n);
    if (rc != GEV_OK) return rc;
    std::vector<double> p(3 * (size_t)n), q(3 * (size_t)n);
    std::vector<int64_t> id((size_t)n);
    int64_t got = 0;
    rc = gev_particles_get(ctx, p.data(), q.data(), id.data(), n, &got);
    if (rc != GEV_OK) return rc;
    // saveGadget2 (Particles_gevolution.hpp:225, :382-385): every tracer_factor-th
    // ID, pos * BoxSize, vel = q / sqrt(a) / GADGET_VELOCITY_CONVERSION / a
    const double rescale_vel = 1.0 / std::sqrt(hdr->time) / 3.335640952e-6;
    std::vector<float> pos, vel;
    std::vector<int64_t> ids;
    pos.reserve(3 * (size_t)got); vel.reserve(3 * (size_t)got); ids.reserve((size_t)got);
    for (int64_t i = 0; i < got; i++) {
        if (id[i] % tracer_factor != 0) continue;
        for (int k = 0; k < 3; k++) {
            pos.push_back((float)(p[3 * i + k] * hdr->BoxSize));
            vel.push_back((float)(q[3 * i + k] * rescale_vel / hdr->time));
        }
        ids.push_back(id[i]);
    }
    return gev_gadget2_write(path, hdr, pos.data(), vel.data(), ids.data(), (int64_t)ids.size());
}

}  // extern "C"
