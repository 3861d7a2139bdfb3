// asset.cpp: the encode's result written as the reference's on-disk asset (src/export.cpp:89-146, 470-812, the layout
// docs/FORMAT.md specifies): level 0's .dds file(s), level 1's .dds and the JSON descriptor.
//
// What has to match the reference byte for byte, and does: the DX10 .dds header (37 little-endian dwords), the level
// order and packing, the uncompressed texel (the index replicated over the byte, a third channel padded to four with
// 255), the BC4/BC5 block bytes and the file split of a block-compressed level 0 (BC4 for one channel, BC5 for two,
// BC5 + BC4 for three, BC5 + BC5 for four). The JSON carries every key a reader needs with the reference's names and
// values; its prose fields ("sampling", "texel", "note", "features") are informational and are this library's own.
//
// Host code only: every input is already on the host (the encode's downloads), and the work is a few bytes per texel.

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "bc.cuh"
#include "device.cuh"

namespace nb
{
namespace
{

constexpr int BLOCK = 4;             // level 1's texel covers BLOCK x BLOCK of level 0's
constexpr int LOD_BIAS_LEVEL1 = 2;   // log2(BLOCK)

int io_error(const std::string& what)
{
    set_error(NNTC_B200_ERR_IO, what);
    return NNTC_B200_ERR_IO;
}

int arg_error(const std::string& what)
{
    set_error(NNTC_B200_ERR_ARG, what);
    return NNTC_B200_ERR_ARG;
}

std::string base_name(const std::string& path)
{
    const size_t slash = path.find_last_of("/\\");
    return slash == std::string::npos ? path : path.substr(slash + 1);
}

// One .dds file: the DX10 header, then the levels base first with nothing between them. size_field is the base level's
// row pitch (uncompressed) or its byte size (block-compressed), and the header's flags say which.
int write_dds(const std::string& path, int w, int h, uint32_t dxgi, bool compressed, uint32_t size_field,
              const std::vector<std::vector<uint8_t>>& levels, size_t& bytes)
{
    const bool chain = levels.size() > 1;
    uint32_t hd[37] = {};
    hd[0] = 0x20534444u;   // "DDS "
    hd[1] = 124;           // the header's own size
    // CAPS | HEIGHT | WIDTH | PIXELFORMAT; MIPMAPCOUNT only for a chain; LINEARSIZE or PITCH for size_field's meaning
    hd[2] = 0x1007u | (chain ? 0x20000u : 0u) | (compressed ? 0x80000u : 0x8u);
    hd[3] = (uint32_t)h;
    hd[4] = (uint32_t)w;
    hd[5] = size_field;
    hd[6] = 1;                                 // depth
    hd[7] = (uint32_t)levels.size();           // stored levels, the base included
    hd[19] = 32;                               // pixel format: its size,
    hd[20] = 0x4u;                             // FOURCC,
    hd[21] = 0x30315844u;                      // "DX10"
    hd[27] = chain ? 0x401008u : 0x1000u;      // TEXTURE, and MIPMAP | COMPLEX for a chain
    hd[32] = dxgi;                             // DX10 extension: the format,
    hd[33] = 3;                                // TEXTURE2D,
    hd[35] = 1;                                // one array slice
    uint8_t le[148];
    for (int i = 0; i < 37; i++)
        for (int b = 0; b < 4; b++)
            le[4 * i + b] = (uint8_t)(hd[i] >> (8 * b));   // little-endian whatever the host
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f)
        return io_error("cannot open '" + path + "' for writing");
    bool ok = std::fwrite(le, 1, sizeof(le), f) == sizeof(le);
    bytes = sizeof(le);
    for (const std::vector<uint8_t>& lv : levels)
    {
        ok = ok && std::fwrite(lv.data(), 1, lv.size(), f) == lv.size();
        bytes += lv.size();
    }
    if (std::fclose(f) != 0)
        ok = false;
    if (!ok)
        return io_error("writing '" + path + "' failed (short write or failed close)");
    return NNTC_B200_OK;
}

// A float the way the descriptor carries it: nine significant digits, enough for any float to read back exactly.
std::string num(double x)
{
    char b[40];
    std::snprintf(b, sizeof(b), "%.9g", x);
    return b;
}

std::string nums(const float* v, int n)
{
    std::string s = "[";
    for (int i = 0; i < n; i++)
        s += (i ? "," : "") + num(v[i]);
    return s + "]";
}

std::string ints(const int* v, int n)
{
    std::string s = "[";
    for (int i = 0; i < n; i++)
        s += (i ? "," : "") + std::to_string(v[i]);
    return s + "]";
}

bool finite_all(const float* v, int n)
{
    for (int i = 0; i < n; i++)
        if (!std::isfinite(v[i]))
            return false;
    return true;
}

// A plane of indices as the bytes an uncompressed file stores: each index replicated over its byte, `stored` bytes a
// texel (a three-channel plane is stored as four, the fourth 255).
std::vector<uint8_t> index_bytes(const uint8_t* k, size_t texels, int channels, int stored, const int* bits)
{
    std::vector<uint8_t> out(texels * (size_t)stored, 255);
    for (size_t t = 0; t < texels; t++)
        for (int c = 0; c < channels; c++)
            out[t * stored + c] = (uint8_t)rep_index(k[t * channels + c], bits[c]);
    return out;
}

// One BC4 block's eight bytes from two endpoints and sixteen 3-bit selectors, packed LSB-first.
void put_bc4(uint8_t* blk, int r0, int r1, const uint8_t sel[16])
{
    blk[0] = (uint8_t)r0;
    blk[1] = (uint8_t)r1;
    uint64_t bits = 0;
    for (int t = 0; t < 16; t++)
        bits |= (uint64_t)(sel[t] & 7) << (3 * t);
    for (int i = 0; i < 6; i++)
        blk[2 + i] = (uint8_t)(bits >> (8 * i));
}

// The channels a block-compressed level-0 file holds: file 0 takes channels 0-1 (or channel 0 alone at C0 = 1), file 1
// the rest.
int file_channels(int c0, int f)
{
    return f == 0 ? (c0 == 1 ? 1 : 2) : c0 - 2;
}

}   // namespace
}   // namespace nb

using namespace nb;

extern "C" int nntc_b200_write_asset(const nntc_b200_model* m, const uint8_t* const* k0, const uint8_t* const* k1,
                                     const uint8_t* const* ep, const uint8_t* const* sel, int source_width,
                                     int source_height, const char* prefix, const char* json_path, size_t* sizes)
{
    if (!m || !k1 || !prefix)
        return arg_error("write_asset: the model, level 1's indices and the prefix are required");
    NB_TRY(validate_model(m));
    const int np = m->nplanes, c0 = m->c0, c1 = m->c1, nout = m->nout, nin = m->nin;
    const bool compress = m->bc0 != 0;
    if (!m->has_decoder)
        return arg_error("write_asset: the model has no decoder to publish");
    // A non-finite number would be written as a token no JSON parser reads: refuse the asset instead.
    if (!finite_all(m->dec_w, nout * nin) || !finite_all(m->dec_b, nout) || !finite_all(m->lo1, c1) ||
        !finite_all(m->hi1, c1) || (m->l0_bc8 && (!finite_all(m->lo0, c0) || !finite_all(m->hi0, c0))))
        return arg_error("write_asset: the decoder or a latent's grid holds a value that is not finite");
    if (source_width < 1 || source_height < 1 || source_width > m->width || source_height > m->height)
        return arg_error("write_asset: the source extent must be positive and within the decoded extent");
    for (int i = 0; i < np; i++)
    {
        if (!k1[i])
            return arg_error("write_asset: level 1's indices of plane " + std::to_string(i) + " are missing");
        const bool blocks = compress && ep && sel && ep[i] && sel[i];
        if (!blocks && (!k0 || !k0[i]))
            return arg_error("write_asset: plane " + std::to_string(i) + " has neither level 0's indices nor its blocks");
    }
    for (int c = 0; c < c0; c++)
        if (m->bits0[c] < 1 || m->bits0[c] > 8)
            return arg_error("write_asset: level 0's bits per channel must be 1..8");
    for (int i = 0; i < np && k0; i++)
        if (k0[i] && !(compress && ep && sel && ep[i] && sel[i]))
            for (size_t t = 0; t < (size_t)m->w0[i] * m->h0[i] * c0; t++)
                if (k0[i][t] > (1 << m->bits0[t % c0]) - 1)
                    return arg_error("write_asset: a level-0 index of plane " + std::to_string(i) +
                                     " is above its channel's bits");
    if (m->bits1 < 4 || m->bits1 > 8)
        return arg_error("write_asset: level 1's bits per channel must be 4..8");

    const std::string pre(prefix);
    const std::string jpath = json_path ? std::string(json_path) : pre + "_nntc.json";
    size_t out_sizes[3] = { 0, 0, 0 };
    std::string mips[2];
    for (int l = 0; l < 2; l++)
    {
        mips[l] = "[";
        for (int i = 0; i < np; i++)
            mips[l] += (i ? ",[" : "[") + std::to_string(l ? m->w1[i] : m->w0[i]) + "," +
                       std::to_string(l ? m->h1[i] : m->h0[i]) + "]";
        mips[l] += "]";
    }

    // ---- level 1: uncompressed, the replicated index; every index must read back as itself on the published grid
    std::string js_l1;
    {
        const int stored = c1 == 3 ? 4 : c1;
        int bits[NNTC_B200_MAX_CHANNELS];
        for (int c = 0; c < c1; c++)
            bits[c] = m->bits1;
        // whether index k of channel c reads back as itself: a property of (c, k) alone, so it is settled once per
        // value and looked up per texel
        bool reads_back[NNTC_B200_MAX_CHANNELS][256];
        for (int c = 0; c < c1; c++)
            for (int k = 0; k < 256; k++)
                reads_back[c][k] =
                    k <= (1 << m->bits1) - 1 &&
                    grid_index(m->lo1[c], m->hi1[c], m->bits1, grid_value(m->lo1[c], m->hi1[c], m->bits1, k)) == k;
        std::vector<std::vector<uint8_t>> levels((size_t)np);
        for (int i = 0; i < np; i++)
        {
            const size_t texels = (size_t)m->w1[i] * m->h1[i];
            for (size_t t = 0; t < texels * c1; t++)
            {
                const int c = (int)(t % c1), k = k1[i][t];
                if (!reads_back[c][k])
                    return arg_error("write_asset: level-1 index " + std::to_string(k) + " of channel " +
                                     std::to_string(c) + " does not read back as itself on its published grid");
            }
            levels[(size_t)i] = index_bytes(k1[i], texels, c1, stored, bits);
        }
        const int dxgi = c1 == 1 ? 61 : (c1 == 2 ? 49 : 28);
        const char* fmt = c1 == 1 ? "R8_UNORM" : (c1 == 2 ? "R8G8_UNORM" : "R8G8B8A8_UNORM");
        const std::string file = pre + "_lat1.dds";
        NB_TRY(write_dds(file, m->w1[0], m->h1[0], (uint32_t)dxgi, false, (uint32_t)(m->w1[0] * stored), levels,
                         out_sizes[1]));
        js_l1 = "    {\n      \"file\": \"" + base_name(file) + "\", \"level\": 1, \"width\": " + std::to_string(m->w1[0]) +
                ", \"height\": " + std::to_string(m->h1[0]) + ",\n      \"dxgi_format\": \"" + fmt +
                "\", \"dxgi_format_id\": " + std::to_string(dxgi) + ", \"channels_used\": " + std::to_string(c1) +
                ", \"channels_stored\": " + std::to_string(stored) + ",\n      \"bits_per_channel\": " +
                ints(bits, c1) + ",\n      \"mip_count\": " + std::to_string(np) + ", \"mip_sizes\": " + mips[1] +
                ",\n      \"texel\": \"uncompressed; each stored byte is the quantisation index k in its top bits, "
                "repeated into the lower bits, so k = byte >> (8 - bits)\",\n      \"dequantise\": { \"kind\": "
                "\"range\", \"note\": \"value = lo + (byte / 255) * (hi - lo), per channel\", \"lo\": " +
                nums(m->lo1, c1) + ", \"hi\": " + nums(m->hi1, c1) + ", \"levels\": " +
                std::to_string((1 << m->bits1) - 1) + " }\n    }\n";
    }

    // ---- level 0
    std::string js_l0;
    {
        const int w = m->w0[0], h = m->h0[0];
        std::string head, fmt_name, texel;
        int dxgi = 0, stored_out = 0;
        if (compress)
        {
            const int nfiles = c0 <= 2 ? 1 : 2;
            std::string files;
            for (int f = 0; f < nfiles; f++)
            {
                const int nc = file_channels(c0, f), bpb = nc == 1 ? 8 : 16;
                std::vector<std::vector<uint8_t>> levels((size_t)np);
                for (int i = 0; i < np; i++)
                {
                    const int pw = m->w0[i], ph = m->h0[i], bx = (pw + 3) / 4, by = (ph + 3) / 4;
                    std::vector<uint8_t>& out = levels[(size_t)i];
                    out.assign((size_t)bx * by * bpb, 0);
                    const bool refined = ep && sel && ep[i] && sel[i];
                    for (int c = 0; c < nc; c++)
                    {
                        const int ch = 2 * f + c;
                        for (int b = 0; b < bx * by; b++)
                        {
                            uint8_t* blk = out.data() + (size_t)b * bpb + (size_t)c * 8;
                            const size_t slot = (size_t)b * c0 + ch;
                            if (refined)
                            {
                                // the blocks the refinement chose are the file
                                put_bc4(blk, ep[i][slot * 2], ep[i][slot * 2 + 1], sel[i] + slot * 16);
                                continue;
                            }
                            // no refined blocks: the seed pack of the stored bytes, the block's edge texels repeated
                            const int gx = b % bx, gy = b / bx;
                            uint8_t v[16];
                            for (int t = 0; t < 16; t++)
                            {
                                const int px = std::min(pw - 1, gx * 4 + t % 4), py = std::min(ph - 1, gy * 4 + t / 4);
                                v[t] = (uint8_t)rep_index(k0[i][((size_t)py * pw + px) * c0 + ch], m->bits0[ch]);
                            }
                            int r0, r1;
                            uint8_t s[16];
                            bc4_seed_block(v, m->bits0[ch], r0, r1, s);
                            put_bc4(blk, r0, r1, s);
                        }
                    }
                }
                const std::string file = pre + "_lat0" + (nfiles == 2 ? (f == 0 ? "a" : "b") : "") + ".dds";
                const int fdx = nc == 1 ? 80 : 83;
                size_t bytes = 0;
                NB_TRY(write_dds(file, w, h, (uint32_t)fdx, true, (uint32_t)levels[0].size(), levels, bytes));
                out_sizes[0] += bytes;
                if (nfiles == 2)
                    files += std::string(f ? ", " : "") + "{ \"file\": \"" + base_name(file) + "\", \"dxgi_format\": \"" +
                             (nc == 1 ? "BC4_UNORM" : "BC5_UNORM") + "\", \"dxgi_format_id\": " + std::to_string(fdx) +
                             ", \"channels_stored\": " + std::to_string(nc) + " }";
                else
                    files = "\"" + base_name(file) + "\"";
            }
            head = nfiles == 2 ? "\"files\": [" + files + "]" : "\"file\": " + files;
            dxgi = file_channels(c0, 0) == 1 ? 80 : 83;
            fmt_name = dxgi == 80 ? "BC4_UNORM" : "BC5_UNORM";
            stored_out = file_channels(c0, 0);
            texel = std::string("BC4 blocks of 4x4 texels per channel (a BC5 block is two channels' BC4 blocks in a row): ") +
                    "two endpoint bytes, then sixteen 3-bit selectors LSB-first in row order, decoded on the standard " +
                    "palette" + (m->l0_bc8 ? "; the blocks were refined against the decoder's output, so the sampled "
                                              "byte is dequantised as it stands"
                                            : "") +
                    (nfiles == 2 ? (c0 == 3 ? "; channels 0-1 are the first file (BC5), channel 2 the second (BC4)"
                                            : "; channels 0-1 are the first file, 2-3 the second (both BC5)")
                                 : "");
        }
        else
        {
            const int stored = c0 == 3 ? 4 : c0;
            std::vector<std::vector<uint8_t>> levels((size_t)np);
            for (int i = 0; i < np; i++)
                levels[(size_t)i] = index_bytes(k0[i], (size_t)m->w0[i] * m->h0[i], c0, stored, m->bits0);
            dxgi = c0 == 1 ? 61 : (c0 == 2 ? 49 : 28);
            fmt_name = c0 == 1 ? "R8_UNORM" : (c0 == 2 ? "R8G8_UNORM" : "R8G8B8A8_UNORM");
            stored_out = stored;
            const std::string file = pre + "_lat0.dds";
            NB_TRY(write_dds(file, w, h, (uint32_t)dxgi, false, (uint32_t)(w * stored), levels, out_sizes[0]));
            head = "\"file\": \"" + base_name(file) + "\"";
            texel = "uncompressed; each stored byte is the quantisation index k in its top bits, repeated into the lower "
                    "bits, so k = byte >> (8 - bits)";
        }
        std::string deq;
        if (m->l0_bc8)
            deq = "{ \"kind\": \"range\", \"note\": \"value = lo + (byte / 255) * (hi - lo), per channel, on the byte the "
                  "block decodes to\", \"lo\": " +
                  nums(m->lo0, c0) + ", \"hi\": " + nums(m->hi0, c0) + ", \"levels\": 255 }";
        else
        {
            // the palette of the shipped format: index k of b bits is -1 + 2 k / (2^b - 1) under the standard BC
            // palette, -1 + 2 rep(k) / 255 on a replicated byte (src/model.h:205-222)
            std::string pal = "[", lo = "[", hi = "[";
            int lv[NNTC_B200_MAX_CHANNELS];
            for (int c = 0; c < c0; c++)
            {
                const int levels = (1 << m->bits0[c]) - 1;
                lv[c] = levels;
                std::vector<float> p((size_t)levels + 1);
                for (int k = 0; k <= levels; k++)
                {
                    const double frac =
                        compress ? (double)k / (double)levels : (double)rep_index(k, m->bits0[c]) / 255.0;
                    p[(size_t)k] = (float)(-1.0 + 2.0 * frac);
                }
                pal += (c ? "," : "") + nums(p.data(), levels + 1);
                lo += (c ? "," : "") + num(p.front());
                hi += (c ? "," : "") + num(p.back());
            }
            deq = "{ \"kind\": \"palette\", \"note\": \"value = palette[c][byte >> (8 - bits)], which equals lo + "
                  "(byte / 255) * (hi - lo) on the byte the sampler returns\", \"palette\": " +
                  pal + "], \"lo\": " + lo + "], \"hi\": " + hi + "], \"levels\": " + ints(lv, c0) + " }";
        }
        js_l0 = "    {\n      " + head + ", \"level\": 0, \"width\": " + std::to_string(w) + ", \"height\": " +
                std::to_string(h) + ",\n      \"dxgi_format\": \"" + fmt_name + "\", \"dxgi_format_id\": " +
                std::to_string(dxgi) + ", \"channels_used\": " + std::to_string(c0) + ", \"channels_stored\": " +
                std::to_string(stored_out) + ",\n" + (compress ? "      \"bc_palette\": \"standard\",\n" : "") +
                "      \"bits_per_channel\": " + ints(m->bits0, c0) + ",\n      \"mip_count\": " + std::to_string(np) +
                ", \"mip_sizes\": " + mips[0] + ",\n      \"texel\": \"" + texel + "\",\n      \"dequantise\": " + deq +
                "\n    },\n";
    }

    // ---- the descriptor
    std::string js = "{\n  \"format\": \"nntc-dds-1\",\n";
    js += "  \"source\": { \"width\": " + std::to_string(source_width) + ", \"height\": " + std::to_string(source_height);
    if (source_width != m->width || source_height != m->height)
        js += ", \"padded\": true, \"padded_width\": " + std::to_string(m->width) + ", \"padded_height\": " +
              std::to_string(m->height);
    js += " },\n";
    js += "  \"decode\": { \"width\": " + std::to_string(m->width) + ", \"height\": " + std::to_string(m->height) +
          ", \"textures_out\": " + std::to_string(m->textures) + " },\n";
    js += "  \"block\": " + std::to_string(BLOCK) + ",\n  \"lod_bias_level1\": " + std::to_string(LOD_BIAS_LEVEL1) + ",\n";
    js += "  \"sampling\": \"sample both textures with the same filter at the same coordinate, level 1 with its UV "
          "gradients scaled by 2^lod_bias_level1 (output mip m reads mip m of both); dequantise each sample after the "
          "filter, then apply the decoder\",\n";
    js += "  \"textures\": [\n" + js_l0 + js_l1 + "  ],\n";
    js += "  \"decoder\": {\n    \"type\": \"bilinear\",\n    \"terms\": \"a b sc\", \"C0\": " + std::to_string(c0) +
          ", \"C1\": " + std::to_string(c1) + ",\n";
    js += "    \"features\": \"phi = [level-1 channels j < C1] [level-0 channels i < C0] [s_i c_j, i outer, j inner]; "
          "out = W phi + b\",\n";
    js += "    \"nin\": " + std::to_string(nin) + ", \"nout\": " + std::to_string(nout) +
          ", \"hidden\": [], \"activation\": \"leaky_relu\", \"leak\": 0,\n    \"output\": \"identity\",\n";
    js += "    \"layers\": [\n      { \"rows\": " + std::to_string(nout) + ", \"cols\": " + std::to_string(nin) +
          ", \"weights\": " + nums(m->dec_w, nout * nin) + ", \"bias\": " + nums(m->dec_b, nout) + " }\n    ]\n  }\n}\n";
    FILE* jf = std::fopen(jpath.c_str(), "wb");
    if (!jf)
        return io_error("cannot open '" + jpath + "' for writing");
    const bool jok = std::fwrite(js.data(), 1, js.size(), jf) == js.size();
    if (std::fclose(jf) != 0 || !jok)
        return io_error("writing '" + jpath + "' failed (short write or failed close)");
    out_sizes[2] = js.size();
    if (sizes)
        std::memcpy(sizes, out_sizes, sizeof(out_sizes));
    return NNTC_B200_OK;
}
