// kdump.h — the KDMP v2 header (koral/io/dump.zig:29-103): a 44-byte
// little-endian record, magic "KDMP", version 2, nx ny nz nv (u32), t (f64),
// nstep (u64), out_idx (u32). Host code shared by the engine's C ABI and the
// oracle. The byte layout is the reference's file format, kept as is so that
// checkpoints move between the two.
#pragma once
#include <stdint.h>
#include <string.h>

#include "../koralcuda.h"

static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "KDMP fields are stored in host order");

namespace kdump {

inline int write_header(const kc_dump_header& h, uint8_t* out) {
  uint32_t ver = KC_KDMP_VERSION;
  memcpy(out, "KDMP", 4);
  memcpy(out + 4, &ver, 4);
  memcpy(out + 8, &h.nx, 4);
  memcpy(out + 12, &h.ny, 4);
  memcpy(out + 16, &h.nz, 4);
  memcpy(out + 20, &h.nv, 4);
  memcpy(out + 24, &h.t, 8);
  memcpy(out + 32, &h.nstep, 8);
  memcpy(out + 40, &h.out_idx, 4);
  return KC_KDMP_HEADER_SIZE;
}

// parseDumpHeader's checks, in its order: length, magic, version
inline int parse_header(const uint8_t* b, int64_t len, kc_dump_header& h) {
  if (!b || len < KC_KDMP_HEADER_SIZE) return KC_ERR_KDMP_TRUNCATED;
  if (memcmp(b, "KDMP", 4) != 0) return KC_ERR_KDMP_BAD_MAGIC;
  uint32_t ver;
  memcpy(&ver, b + 4, 4);
  if (ver != KC_KDMP_VERSION) return KC_ERR_KDMP_BAD_VERSION;
  memcpy(&h.nx, b + 8, 4);
  memcpy(&h.ny, b + 12, 4);
  memcpy(&h.nz, b + 16, 4);
  memcpy(&h.nv, b + 20, 4);
  memcpy(&h.t, b + 24, 8);
  memcpy(&h.nstep, b + 32, 8);
  memcpy(&h.out_idx, b + 40, 4);
  return KC_OK;
}

inline int64_t body_bytes(int64_t nx, int64_t ny, int64_t nz, int64_t nv) { return nx * ny * nz * nv * 8; }

}  // namespace kdump
