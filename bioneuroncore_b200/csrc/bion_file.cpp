// bion_file.cpp -- .bion files: the reader for every version the reference's loaders
// accept (3-14) and the version-14 writer.
//
// The reference reads a .bion with bion_load_host (src/bion_loader_host.cpp:26-428) on
// its CPU path and with bion_load_cuda (src/bion_loader.cpp:634-982) in its GPU backend.
// Both take the layout of each record from the header's version and, from version 10
// on, from the record sizes the header declares (include/bion_format.h:59-340):
//
//   header      68 bytes (v3-v4), 84 (v5-v9: + nucleus count and version), 100 (v10+:
//               + the file_sz_* record sizes)
//   neuron      24 bytes, every version
//   segment     852 (v3), 1692 (v4-v6, read with 88-byte modifiers), 1692 (v7-v9),
//               v10+: 1692 / 1696 / 1704 / 3208 / 3216 by file_sz_segment
//   connection  12 bytes with a coupling resistance (v3-v8), 16 (v9+)
//   synapse     824 (v3-v6), 836 (v7-v9), v10+: 836 / 1560 / 1568 by file_sz_synapse
//   nucleus     204 (v5), 332 (v6), v7+: 412 (46 genes) by file_sz_nucleus, else 500
//
// Each old layout is restated below as byte offsets into the record (the offsets are
// the file format); the conversions follow the reference's migration functions field
// by field, including where those read neighbouring fields: a v7-v9 segment carries
// five ions per side, and its migration copies seven, so ions 5 and 6 take the floats
// that follow each array.  Versions 4-6 are read as the reference reads them: 196 bytes
// copied over the start of the current record, then 88-byte modifiers.  Where the
// reference leaves bytes of a record unwritten (new[] memory that no assignment
// reaches: a v3-v6 synapse past its 824 bytes, a v3-v8 connection's reserved bytes, a
// v6 nucleus past its 332 bytes) this reader writes zeros.
//
// A file without nucleus records gets one default nucleus per neuron (id of the neuron,
// enabled, consolidation mode 3, amino-acid level 0.5), as both reference loaders
// create them (bion_loader_host.cpp:340-353, bion_loader.cpp:902-914).  The reference's
// GPU backend maps protein levels onto synapse parameters from those
// (gpu_backend_cuda.cu:275-289).
#include "bion_file.h"

#include <cstdio>
#include <cstring>
#include <ctime>
#include <new>
#include <vector>

namespace bnc {
namespace {

constexpr uint32_t kMagic = 0x42494F4Eu;
constexpr size_t kHdrV3 = 68, kHdrV5 = 84, kHdrV10 = 100;
constexpr size_t kSegV3 = 852, kSegV4 = 1692, kSegV7 = 1692, kSegV7Er = 1696, kSegV10 = 1704, kSegV13 = 3208;
constexpr size_t kSynV6 = 824, kSynV7 = 836, kSynV13 = 1560;
constexpr size_t kNuc = 500, kNucV46 = 412, kNucV6 = 332, kNucV5 = 204;
constexpr size_t kModV3 = 41, kModV12 = 44, kMod = sizeof(BncModifier);

// Current nucleus record (types.h:508-524 with 57 genes): offsets used here.
constexpr size_t kNucGene = 16, kNucProtein = 244, kNucTail = 472, kNucAmino = 492;

template <class T>
T rd(const uint8_t* p, size_t off) {
    T v;
    std::memcpy(&v, p + off, sizeof(T));
    return v;
}
template <class T>
void wr(uint8_t* p, size_t off, T v) {
    std::memcpy(p + off, &v, sizeof(T));
}

// v3 modifier, 41 bytes: type, float density, float state[8], active_vars, flags.
void mod_from_v3(const uint8_t* m, BncModifier* s) {
    s->type = m[0];
    s->density = rd<float>(m, 1);
    for (int k = 0; k < 8; k++) s->state[k] = rd<float>(m, 5 + 4 * k);
    s->active_vars = m[37];
    s->flags = m[38];
}

// v4-v12 modifier, 44 bytes (bion_migrate_modifier_v12, bion_format.h:59-78).
void mod_from_v12(const uint8_t* m, BncModifier* s) {
    s->type = m[0];
    s->density = rd<float>(m, 4);
    for (int k = 0; k < 8; k++) s->state[k] = rd<float>(m, 8 + 4 * k);
    s->active_vars = m[40];
    s->flags = m[41];
}

void seg_head(const uint8_t* r, BncSegment* s) {   // id .. radius: the same bytes in every layout
    s->id = rd<uint32_t>(r, 0);
    s->neuron_id = rd<uint32_t>(r, 4);
    std::memcpy(&s->position, r + 8, 12);
    std::memcpy(&s->direction, r + 20, 12);
    s->length = rd<float>(r, 32);
    s->radius = rd<float>(r, 36);
}

void seg_ids(const uint8_t* r, size_t off, BncSegment* s) {
    for (int j = 0; j < 16; j++) s->intra_connection_ids[j] = rd<uint32_t>(r, off + 4 * j);
}

// v3 (bion_loader_host.cpp:146-210): no direction, 4 ions, 12 transmitters.
void seg_from_v3(const uint8_t* r, BncSegment* s) {
    std::memset(s, 0, sizeof(*s));
    s->id = rd<uint32_t>(r, 0);
    s->neuron_id = rd<uint32_t>(r, 4);
    std::memcpy(&s->position, r + 8, 12);
    s->direction.x = 0.0f; s->direction.y = 1.0f; s->direction.z = 0.0f;
    s->length = rd<float>(r, 20);
    s->radius = rd<float>(r, 24);
    s->V_m = rd<float>(r, 28);
    for (int j = 0; j < 4; j++) {
        s->intra_ions[j] = rd<float>(r, 32 + 4 * j);
        s->extra_ions[j] = rd<float>(r, 48 + 4 * j);
    }
    for (int j = 0; j < 12; j++) s->neurotransmitter[j] = rd<float>(r, 64 + 4 * j);
    s->modifier_count = r[768];
    s->segment_type = 0;
    s->ATP_level = rd<float>(r, 772);
    s->temperature = rd<float>(r, 776);
    s->I_buffer = rd<float>(r, 780);
    seg_ids(r, 784, s);
    s->intra_connection_count = r[848];
    // The reference converts modifier_count modifiers without a bound; the record holds
    // 16 and the current one 32 (a count above 32 is then refused by validation), so
    // slots past the record's 16 stay zero here.
    for (int j = 0; j < s->modifier_count && j < 16; j++) mod_from_v3(r + 112 + kModV3 * j, &s->modifiers[j]);
}

// v4-v6 (bion_loader_host.cpp:104-145): the first 196 bytes copied over the current
// record as they are, then up to 16 modifiers of 88 bytes, then the tail fields.
void seg_from_v4(const uint8_t* r, BncSegment* s) {
    std::memset(s, 0, sizeof(*s));
    std::memcpy(s, r, 196);
    int n = r[1604];
    if (n > 16) n = 16;
    s->modifier_count = (uint8_t)n;
    for (int j = 0; j < n; j++) std::memcpy(&s->modifiers[j], r + 196 + kMod * j, kMod);
    s->segment_type = r[1605];
    s->ATP_level = rd<float>(r, 1608);
    s->temperature = rd<float>(r, 1612);
    s->I_buffer = rd<float>(r, 1616);
    s->transcription_signal = rd<float>(r, 1620);
    seg_ids(r, 1624, s);
    s->intra_connection_count = r[1688];
}

// v7-v9 and early v10 (bion_migrate_segment_v7, bion_format.h:446-475): 14
// transmitters, 44-byte modifiers; er_ca2 from the 4 bytes after a 1696-byte record.
void seg_from_v7(const uint8_t* r, BncSegment* s, float er_ca2) {
    std::memset(s, 0, sizeof(*s));
    seg_head(r, s);
    s->V_m = rd<float>(r, 40);
    for (int j = 0; j < 7; j++) {   // seven ions from five-element arrays (see the header)
        s->intra_ions[j] = rd<float>(r, 44 + 4 * j);
        s->extra_ions[j] = rd<float>(r, 64 + 4 * j);
    }
    for (int j = 0; j < 14; j++) {
        s->intra_nt[j] = rd<float>(r, 84 + 4 * j);
        s->neurotransmitter[j] = rd<float>(r, 140 + 4 * j);
    }
    int n = r[1604];
    if (n > 32) n = 32;
    s->modifier_count = (uint8_t)n;
    for (int j = 0; j < n; j++) mod_from_v12(r + 196 + kModV12 * j, &s->modifiers[j]);
    s->segment_type = r[1605];
    s->ATP_level = rd<float>(r, 1608);
    s->temperature = rd<float>(r, 1612);
    s->I_buffer = rd<float>(r, 1616);
    s->transcription_signal = rd<float>(r, 1620);
    seg_ids(r, 1624, s);
    s->intra_connection_count = r[1688];
    s->ER_Ca2 = er_ca2;
}

// v10 with 1704-byte records (bion_migrate_segment_v10, bion_format.h:311-340): 5 ions,
// 15 transmitters, 44-byte modifiers, ER_Ca2.
void seg_from_v10(const uint8_t* r, BncSegment* s) {
    std::memset(s, 0, sizeof(*s));
    seg_head(r, s);
    s->V_m = rd<float>(r, 40);
    for (int j = 0; j < 5; j++) {
        s->intra_ions[j] = rd<float>(r, 44 + 4 * j);
        s->extra_ions[j] = rd<float>(r, 64 + 4 * j);
    }
    for (int j = 0; j < 15; j++) {
        s->intra_nt[j] = rd<float>(r, 84 + 4 * j);
        s->neurotransmitter[j] = rd<float>(r, 144 + 4 * j);
    }
    int n = r[1612];
    if (n > 32) n = 32;
    s->modifier_count = (uint8_t)n;
    for (int j = 0; j < n; j++) mod_from_v12(r + 204 + kModV12 * j, &s->modifiers[j]);
    s->segment_type = r[1613];
    s->ATP_level = rd<float>(r, 1616);
    s->temperature = rd<float>(r, 1620);
    s->I_buffer = rd<float>(r, 1624);
    s->transcription_signal = rd<float>(r, 1628);
    seg_ids(r, 1632, s);
    s->intra_connection_count = r[1696];
    s->ER_Ca2 = rd<float>(r, 1700);
}

// v13, 3208 bytes (bion_migrate_segment_v13, bion_format.h:374-406): the current fields
// with I_buffer 4 bytes earlier.
void seg_from_v13(const uint8_t* r, BncSegment* s) {
    std::memset(s, 0, sizeof(*s));
    seg_head(r, s);
    s->V_m = rd<double>(r, 40);
    for (int j = 0; j < 8; j++) {
        s->intra_ions[j] = rd<double>(r, 48 + 8 * j);
        s->extra_ions[j] = rd<double>(r, 112 + 8 * j);
    }
    for (int j = 0; j < 15; j++) {
        s->intra_nt[j] = rd<float>(r, 176 + 4 * j);
        s->neurotransmitter[j] = rd<float>(r, 236 + 4 * j);
    }
    int n = r[3112];
    if (n > 32) n = 32;
    s->modifier_count = (uint8_t)n;
    for (int j = 0; j < n; j++) std::memcpy(&s->modifiers[j], r + 296 + kMod * j, kMod);
    s->segment_type = r[3113];
    s->ATP_level = rd<float>(r, 3116);
    s->temperature = rd<float>(r, 3120);
    s->I_buffer = rd<double>(r, 3124);
    s->transcription_signal = rd<float>(r, 3132);
    seg_ids(r, 3136, s);
    s->intra_connection_count = r[3200];
    s->ER_Ca2 = rd<float>(r, 3204);
}

// Records of another declared size (bion_read_sized, bion_format.h:33-48): the common
// prefix copied, the rest zero.
void copy_sized(const uint8_t* r, size_t file_sz, void* dst, size_t code_sz) {
    std::memset(dst, 0, code_sz);
    std::memcpy(dst, r, file_sz < code_sz ? file_sz : code_sz);
}

void syn_head(const uint8_t* r, BncSynapse* s) {
    s->id = rd<uint32_t>(r, 0);
    s->pre_segment = rd<uint32_t>(r, 4);
    s->post_segment = rd<uint32_t>(r, 8);
    s->type = r[12];
    s->weight = rd<float>(r, 16);
    s->delay = rd<float>(r, 20);
    s->pre_area = rd<float>(r, 24);
    s->post_area = rd<float>(r, 28);
}

// v3-v6, 824 bytes (bion_loader_host.cpp:236-249): copied over the start of the current
// record, then the pool fields set.
void syn_from_v6(const uint8_t* r, BncSynapse* s) {
    std::memset(s, 0, sizeof(*s));
    std::memcpy(s, r, kSynV6);
    s->RRP = 10.0f;
    s->RRP_max = 10.0f;
    s->RRP_recovery = 0.02f;
}

// v7-v9 and early v10, 836 bytes (bion_migrate_synapse_v7, bion_format.h:114-146).
void syn_from_v7(const uint8_t* r, BncSynapse* s) {
    std::memset(s, 0, sizeof(*s));
    syn_head(r, s);
    int n = r[384];
    if (n > 8) n = 8;
    s->pre_autoreceptor_count = (uint8_t)n;
    for (int j = 0; j < n; j++) mod_from_v12(r + 32 + kModV12 * j, &s->pre_autoreceptors[j]);
    n = r[740];
    if (n > 8) n = 8;
    s->post_receptor_count = (uint8_t)n;
    for (int j = 0; j < n; j++) mod_from_v12(r + 388 + kModV12 * j, &s->post_receptors[j]);
    s->release_probability = rd<float>(r, 744);
    s->release_amount = rd<float>(r, 748);
    for (int j = 0; j < 14; j++) s->cleft_neurotransmitter[j] = rd<float>(r, 752 + 4 * j);
    s->facilitation = rd<float>(r, 808);
    s->depression = rd<float>(r, 812);
    s->tau_clearance = rd<float>(r, 816);
    s->refractory = r[820];
    s->RRP = rd<float>(r, 824);
    s->RRP_max = rd<float>(r, 828);
    s->RRP_recovery = rd<float>(r, 832);
}

// v13, 1560 bytes (bion_migrate_synapse_v13, bion_format.h:185-220): the current fields
// with the receptor arrays 4 bytes earlier.
void syn_from_v13(const uint8_t* r, BncSynapse* s) {
    std::memset(s, 0, sizeof(*s));
    syn_head(r, s);
    int n = r[736];
    if (n > 8) n = 8;
    s->pre_autoreceptor_count = (uint8_t)n;
    for (int j = 0; j < n; j++) std::memcpy(&s->pre_autoreceptors[j], r + 32 + kMod * j, kMod);
    n = r[1444];
    if (n > 8) n = 8;
    s->post_receptor_count = (uint8_t)n;
    for (int j = 0; j < n; j++) std::memcpy(&s->post_receptors[j], r + 740 + kMod * j, kMod);
    s->release_probability = rd<float>(r, 1448);
    s->release_amount = rd<float>(r, 1452);
    for (int j = 0; j < 15; j++) s->cleft_neurotransmitter[j] = rd<float>(r, 1456 + 4 * j);
    s->facilitation = rd<float>(r, 1516);
    s->depression = rd<float>(r, 1520);
    s->tau_clearance = rd<float>(r, 1524);
    s->refractory = r[1528];
    s->RRP = rd<float>(r, 1532);
    s->RRP_max = rd<float>(r, 1536);
    s->RRP_recovery = rd<float>(r, 1540);
    s->bouton_Ca = rd<float>(r, 1544);
    s->spine_Ca = rd<float>(r, 1548);
    s->spine_camkii = rd<float>(r, 1552);
    s->spine_calcineurin = rd<float>(r, 1556);
}

void nuc_ids(const uint8_t* r, uint8_t* n) {   // neuron id, enabled, mode, interval, last tick
    wr<uint32_t>(n, 0, rd<uint32_t>(r, 0));
    n[4] = r[4];
    n[5] = r[5];
    wr<uint32_t>(n, 8, rd<uint32_t>(r, 8));
    wr<uint32_t>(n, 12, rd<uint32_t>(r, 12));
}

// v5, 204 bytes with 20 genes (bion_loader_host.cpp:268-293).
void nuc_from_v5(const uint8_t* r, uint8_t* n) {
    std::memset(n, 0, kNuc);
    nuc_ids(r, n);
    for (int g = 0; g < 20; g++) {
        wr<float>(n, kNucGene + 4 * g, rd<float>(r, 16 + 4 * g));
        wr<float>(n, kNucProtein + 4 * g, rd<float>(r, 96 + 4 * g));
    }
    std::memcpy(n + kNucTail, r + 176, 24);   // synthesis rate, pCREB, ERK, NF-kB, mTORC1, amino acids
}

// v6, 332 bytes with 36 genes (bion_loader_host.cpp:294-309): copied over the start of
// the current record, then genes 36-45 of both arrays cleared.
void nuc_from_v6(const uint8_t* r, uint8_t* n) {
    std::memset(n, 0, kNuc);
    std::memcpy(n, r, kNucV6);
    for (int g = 36; g < 46; g++) {
        wr<float>(n, kNucGene + 4 * g, 0.0f);
        wr<float>(n, kNucProtein + 4 * g, 0.0f);
    }
}

// 412 bytes with 46 genes (bion_migrate_nucleus_v46, bion_format.h:515-535).
void nuc_from_v46(const uint8_t* r, uint8_t* n) {
    std::memset(n, 0, kNuc);
    nuc_ids(r, n);
    for (int g = 0; g < 46; g++) {
        wr<float>(n, kNucGene + 4 * g, rd<float>(r, 16 + 4 * g));
        wr<float>(n, kNucProtein + 4 * g, rd<float>(r, 200 + 4 * g));
    }
    std::memcpy(n + kNucTail, r + 384, 24);
}

void nuc_default(uint32_t neuron_id, uint8_t* n) {
    std::memset(n, 0, kNuc);
    wr<uint32_t>(n, 0, neuron_id);
    n[4] = 1;   // enabled
    n[5] = 3;   // consolidation and reconsolidation
    wr<float>(n, kNucAmino, 0.5f);
}

// Reads count records of rec_sz bytes and converts each with f(record, index).
template <class F>
bool read_records(FILE* f, uint32_t count, size_t rec_sz, F conv) {
    std::vector<uint8_t> buf(rec_sz);
    for (uint32_t i = 0; i < count; i++) {
        if (fread(buf.data(), rec_sz, 1, f) != 1) return false;
        conv(buf.data(), i);
    }
    return true;
}

int read_segments(FILE* f, BncBionData* d) {
    const uint32_t v = d->header.version, n = d->num_segments, fsz = d->header.file_sz_segment;
    BncSegment* s = d->segments;
    bool ok;
    if (v >= 10 && (fsz == 0 || fsz == sizeof(BncSegment))) {
        ok = fread(s, sizeof(BncSegment), n, f) == n;
    } else if (v >= 10 && fsz == kSegV7Er) {
        ok = read_records(f, n, kSegV7Er, [&](const uint8_t* r, uint32_t i) { seg_from_v7(r, s + i, rd<float>(r, kSegV7)); });
    } else if (v >= 7 && (v < 10 || fsz == kSegV7)) {
        ok = read_records(f, n, kSegV7, [&](const uint8_t* r, uint32_t i) { seg_from_v7(r, s + i, 0.0f); });
    } else if (v >= 10 && fsz == kSegV10) {
        ok = read_records(f, n, kSegV10, [&](const uint8_t* r, uint32_t i) { seg_from_v10(r, s + i); });
    } else if (v >= 10 && fsz == kSegV13) {
        ok = read_records(f, n, kSegV13, [&](const uint8_t* r, uint32_t i) { seg_from_v13(r, s + i); });
    } else if (v >= 10) {
        ok = read_records(f, n, fsz, [&](const uint8_t* r, uint32_t i) { copy_sized(r, fsz, s + i, sizeof(BncSegment)); });
    } else if (v >= 4) {
        ok = read_records(f, n, kSegV4, [&](const uint8_t* r, uint32_t i) { seg_from_v4(r, s + i); });
    } else {
        ok = read_records(f, n, kSegV3, [&](const uint8_t* r, uint32_t i) { seg_from_v3(r, s + i); });
    }
    return ok ? BNC_OK : BNC_BION_ERR_FILE_READ;
}

int read_connections(FILE* f, BncBionData* d) {
    const uint32_t n = d->num_connections;
    if (!n) return BNC_OK;
    BncIntraConnection* c = d->connections;
    bool ok;
    if (d->header.version <= 8) {   // 12 bytes: a coupling resistance, now a flag (bion_loader_host.cpp:212-228)
        ok = read_records(f, n, 12, [&](const uint8_t* r, uint32_t i) {
            std::memset(c + i, 0, sizeof(*c));
            c[i].segment_a = rd<uint32_t>(r, 0);
            c[i].segment_b = rd<uint32_t>(r, 4);
            c[i].is_intracellular = rd<float>(r, 8) != 0.0f ? 1 : 0;
        });
    } else {
        ok = fread(c, sizeof(BncIntraConnection), n, f) == n;
    }
    return ok ? BNC_OK : BNC_BION_ERR_FILE_READ;
}

int read_synapses(FILE* f, BncBionData* d) {
    const uint32_t v = d->header.version, n = d->num_synapses, fsz = d->header.file_sz_synapse;
    if (!n) return BNC_OK;
    BncSynapse* s = d->synapses;
    bool ok;
    if (v <= 6) {
        ok = read_records(f, n, kSynV6, [&](const uint8_t* r, uint32_t i) { syn_from_v6(r, s + i); });
    } else if (v >= 10 && (fsz == 0 || fsz == sizeof(BncSynapse))) {
        ok = fread(s, sizeof(BncSynapse), n, f) == n;
    } else if (v < 10 || fsz == kSynV7) {
        ok = read_records(f, n, kSynV7, [&](const uint8_t* r, uint32_t i) { syn_from_v7(r, s + i); });
    } else if (fsz == kSynV13) {
        ok = read_records(f, n, kSynV13, [&](const uint8_t* r, uint32_t i) { syn_from_v13(r, s + i); });
    } else {
        ok = read_records(f, n, fsz, [&](const uint8_t* r, uint32_t i) { copy_sized(r, fsz, s + i, sizeof(BncSynapse)); });
    }
    return ok ? BNC_OK : BNC_BION_ERR_FILE_READ;
}

int read_nuclei(FILE* f, BncBionData* d, bool default_nuclei) {
    const uint32_t v = d->header.version;
    if (v >= 5 && d->header.num_nuclei > 0) {
        const uint32_t n = d->header.num_nuclei;
        uint8_t* nu = new (std::nothrow) uint8_t[(size_t)n * kNuc];
        if (!nu) return BNC_ERR_ALLOC;
        d->nuclei = nu;
        d->num_nuclei = n;
        bool ok;
        if (v == 5) {
            ok = read_records(f, n, kNucV5, [&](const uint8_t* r, uint32_t i) { nuc_from_v5(r, nu + (size_t)i * kNuc); });
        } else if (v == 6) {
            ok = read_records(f, n, kNucV6, [&](const uint8_t* r, uint32_t i) { nuc_from_v6(r, nu + (size_t)i * kNuc); });
        } else if (d->header.file_sz_nucleus == kNucV46) {
            ok = read_records(f, n, kNucV46, [&](const uint8_t* r, uint32_t i) { nuc_from_v46(r, nu + (size_t)i * kNuc); });
        } else {
            ok = fread(nu, kNuc, n, f) == n;
        }
        return ok ? BNC_OK : BNC_BION_ERR_FILE_READ;
    }
    if (!default_nuclei || d->num_neurons == 0) return BNC_OK;
    uint8_t* nu = new (std::nothrow) uint8_t[(size_t)d->num_neurons * kNuc];
    if (!nu) return BNC_ERR_ALLOC;
    for (uint32_t i = 0; i < d->num_neurons; i++) nuc_default(d->neurons[i].id, nu + (size_t)i * kNuc);
    d->nuclei = nu;
    d->num_nuclei = d->num_neurons;
    return BNC_OK;
}

// The reference loader's checks after reading (bion_loader_host.cpp:359-408), in its
// order, then each segment's incidence list (:410-425).
int validate(BncBionData* d) {
    for (uint32_t i = 0; i < d->num_connections; i++)
        if (d->connections[i].segment_a >= d->num_segments || d->connections[i].segment_b >= d->num_segments) {
            set_error("connection %u: segment out of range", i);
            return BNC_BION_ERR_BAD_CONN;
        }
    for (uint32_t i = 0; i < d->num_synapses; i++) {
        const BncSynapse& y = d->synapses[i];
        if (y.pre_segment >= d->num_segments || y.post_segment >= d->num_segments) {
            set_error("synapse %u: segment out of range", i);
            return BNC_BION_ERR_BAD_SYNAPSE;
        }
        if (y.pre_autoreceptor_count > BNC_MAX_PRE_AUTORECEPTORS || y.post_receptor_count > BNC_MAX_POST_RECEPTORS) {
            set_error("synapse %u: too many receptors", i);
            return BNC_ERR_FORMAT;
        }
        if (y.type >= 3) {
            set_error("synapse %u: invalid type %u", i, (unsigned)y.type);
            return BNC_BION_ERR_BAD_SYNAPSE;
        }
    }
    for (uint32_t i = 0; i < d->num_neurons; i++)
        if ((uint64_t)d->neurons[i].segment_start + d->neurons[i].segment_count > d->num_segments) {
            set_error("neuron %u: segment range past the segments", i);
            return BNC_BION_ERR_BAD_NEURON;
        }
    for (uint32_t i = 0; i < d->num_segments; i++)
        if (d->segments[i].modifier_count > BNC_MAX_MODIFIERS) {
            set_error("segment %u: too many modifiers", i);
            return BNC_ERR_FORMAT;
        }
    for (uint32_t i = 0; i < d->num_segments; i++) d->segments[i].intra_connection_count = 0;
    for (uint32_t i = 0; i < d->num_connections; i++) {
        BncSegment& a = d->segments[d->connections[i].segment_a];
        BncSegment& b = d->segments[d->connections[i].segment_b];
        if (a.intra_connection_count < BNC_MAX_INTRACONN_PER_SEG) a.intra_connection_ids[a.intra_connection_count++] = i;
        if (b.intra_connection_count < BNC_MAX_INTRACONN_PER_SEG) b.intra_connection_ids[b.intra_connection_count++] = i;
    }
    return BNC_OK;
}

}  // namespace

void bion_free(BncBionData& d) {
    delete[] d.neurons;
    delete[] d.segments;
    delete[] d.connections;
    delete[] d.synapses;
    delete[] static_cast<uint8_t*>(d.nuclei);
    std::memset(&d, 0, sizeof(d));
}

int bion_read(const char* path, BncBionData* d, bool default_nuclei) {
    std::memset(d, 0, sizeof(*d));
    FILE* f = fopen(path, "rb");
    if (!f) { set_error("cannot open %s", path); return BNC_BION_ERR_FILE_OPEN; }
    auto fail = [&](int code, const char* msg) {
        fclose(f);
        bion_free(*d);
        set_error("%s: %s", path, msg);
        return code;
    };
    uint8_t* hdr = reinterpret_cast<uint8_t*>(&d->header);
    if (fread(hdr, kHdrV3, 1, f) != 1) return fail(BNC_BION_ERR_FILE_READ, "short header");
    if (d->header.version >= 5) {
        const size_t ext = (d->header.version >= 10 ? kHdrV10 : kHdrV5) - kHdrV3;
        if (fread(hdr + kHdrV3, ext, 1, f) != 1) return fail(BNC_BION_ERR_FILE_READ, "short header");
    }
    if (d->header.magic != kMagic) return fail(BNC_BION_ERR_BAD_MAGIC, "bad magic");
    if (d->header.version < 3 || d->header.version > 14) return fail(BNC_BION_ERR_BAD_VERSION, "unsupported version");
    if (d->header.num_segments == 0) return fail(BNC_BION_ERR_ZERO_SEGS, "zero segments");
    d->num_neurons = d->header.num_neurons;
    d->num_segments = d->header.num_segments;
    d->num_connections = d->header.num_intra_connections;
    d->num_synapses = d->header.num_synapses;
    d->neurons = new (std::nothrow) BncNeuron[d->num_neurons ? d->num_neurons : 1];
    d->segments = new (std::nothrow) BncSegment[d->num_segments];
    d->connections = new (std::nothrow) BncIntraConnection[d->num_connections ? d->num_connections : 1];
    d->synapses = new (std::nothrow) BncSynapse[d->num_synapses ? d->num_synapses : 1];
    if (!d->neurons || !d->segments || !d->connections || !d->synapses) return fail(BNC_ERR_ALLOC, "out of memory");
    if (d->num_neurons && fread(d->neurons, sizeof(BncNeuron), d->num_neurons, f) != d->num_neurons)
        return fail(BNC_BION_ERR_FILE_READ, "short neurons");
    int rc = read_segments(f, d);
    if (rc != BNC_OK) return fail(rc, "short segments");
    rc = read_connections(f, d);
    if (rc != BNC_OK) return fail(rc, "short connections");
    rc = read_synapses(f, d);
    if (rc != BNC_OK) return fail(rc, "short synapses");
    rc = read_nuclei(f, d, default_nuclei);
    if (rc != BNC_OK) return fail(rc, rc == BNC_ERR_ALLOC ? "out of memory" : "short nuclei");
    fclose(f);
    rc = validate(d);
    if (rc != BNC_OK) bion_free(*d);
    return rc;
}

int bion_write(const BncBionData& d, const char* path) {
    FILE* f = fopen(path, "wb");
    if (!f) { set_error("cannot open %s for writing", path); return BNC_BION_ERR_FILE_OPEN; }
    BncNetworkHeader hdr = d.header;
    hdr.magic = kMagic;
    hdr.version = 14;
    hdr.mode = 0;
    hdr.diffusion_type = 0;
    hdr.num_neurons = d.num_neurons;
    hdr.num_segments = d.num_segments;
    hdr.num_intra_connections = d.num_connections;
    hdr.num_synapses = d.num_synapses;
    hdr.grid_dim_x = hdr.grid_dim_y = hdr.grid_dim_z = 0;
    hdr.voxel_size = 1.0f;
    hdr.timestamp = (uint64_t)time(nullptr);
    std::strncpy(hdr.build_id, "v5.0.0", sizeof(hdr.build_id) - 1);
    hdr.num_nuclei = d.nuclei ? d.num_nuclei : 0;
    hdr.nucleus_version = 1;
    hdr.file_sz_segment = sizeof(BncSegment);
    hdr.file_sz_synapse = sizeof(BncSynapse);
    hdr.file_sz_nucleus = kNuc;
    hdr.file_sz_intraconnection = sizeof(BncIntraConnection);
    hdr.file_sz_neuron = sizeof(BncNeuron);
    hdr.file_sz_modifier = sizeof(BncModifier);
    bool ok = fwrite(&hdr, sizeof(hdr), 1, f) == 1;
    if (ok && d.num_neurons) ok = fwrite(d.neurons, sizeof(BncNeuron), d.num_neurons, f) == d.num_neurons;
    if (ok) ok = fwrite(d.segments, sizeof(BncSegment), d.num_segments, f) == d.num_segments;
    if (ok && d.num_connections)
        ok = fwrite(d.connections, sizeof(BncIntraConnection), d.num_connections, f) == d.num_connections;
    if (ok && d.num_synapses) ok = fwrite(d.synapses, sizeof(BncSynapse), d.num_synapses, f) == d.num_synapses;
    if (ok && hdr.num_nuclei) ok = fwrite(d.nuclei, kNuc, hdr.num_nuclei, f) == hdr.num_nuclei;
    fclose(f);
    if (!ok) { set_error("write to %s failed", path); return BNC_BION_ERR_WRITE_FAIL; }
    return BNC_OK;
}

}  // namespace bnc
