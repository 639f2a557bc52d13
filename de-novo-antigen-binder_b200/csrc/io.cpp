// io.cpp — the reference's input and output formats, host C++ behind the C ABI.
//
//  * parse_pdb (pdb.rs:19-57): one residue per ATOM / HETATM record whose atom
//    name (columns 13-16) is CA; residue name columns 18-20
//    (AminoAcid::from_three_letter, atom.rs:127-151: HID/HIE/HIP are His, unknown
//    names Gly); x, y, z columns 31-38, 39-46, 47-54 (an unparsable field reads 0).
//  * parse_peptide (pdb.rs:64-83): one-letter sequence on an extended trace along
//    x, x = (i - n * 0.5) * 3.8 in f32.
//  * write_pdb (pdb.rs:90-114), write_pdb_allatom (pdb.rs:121-152), write_pdb_multi
//    (pdb.rs:157-191): fixed-column ATOM records, serials capped at 99999 and
//    residue numbers at 9999, TER between chains, END.
//  * write_fasta / write_json / write_csv (report.rs:41-113).
//
// Numbers are formatted with the C library's printf, which rounds the exact binary
// value as Rust's fixed-precision formatting does.  Output goes into a caller
// buffer: BINDER_ERR_CAPACITY with *out_len = the bytes needed (without the NUL)
// when it is too small; otherwise the text is NUL-terminated.
#include <cctype>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "binder_gpu.h"

namespace {

#include "binder_tables.inc"

void appendf(std::string& s, const char* fmt, ...) {
    char buf[256];
    va_list ap;
    va_start(ap, fmt);
    const int n = std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (n > 0) s.append(buf, (size_t)std::min(n, (int)sizeof buf - 1));
}

int emit(const std::string& s, char* out, size_t cap, size_t* out_len) {
    if (!out_len) return BINDER_ERR_ARG;
    *out_len = s.size();
    if (!out || cap < s.size() + 1) return BINDER_ERR_CAPACITY;
    std::memcpy(out, s.data(), s.size());
    out[s.size()] = '\0';
    return BINDER_OK;
}

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
}

// line.get(a..b): the columns when the line is long enough, else nothing
bool field(const std::string& line, size_t a, size_t b, std::string& out) {
    if (line.size() < b) return false;
    out = line.substr(a, b - a);
    return true;
}

// str::parse::<f32> of a trimmed field: a complete decimal number, else none
bool parse_f32(const std::string& s, float& v) {
    if (s.empty()) return false;
    const char* p = s.c_str();
    char* end = nullptr;
    const float x = std::strtof(p, &end);
    if (end == p || *end != '\0') return false;
    for (char c : s)  // strtof also takes hexadecimal and "nan"/"inf" spellings Rust does not
        if (c == 'x' || c == 'X' || c == 'p' || c == 'P') return false;
    v = x;
    return true;
}

int aa_from_three(const std::string& s) {
    if (s == "HID" || s == "HIE" || s == "HIP") return 8;  // His
    for (int a = 0; a < 20; ++a)
        if (s == BT_AA3[a]) return a;
    return 7;  // Gly
}

int aa_from_one(char c) {
    static const char ONE[] = "ARNDCQEGHILKMFPSTWYV";
    c = (char)std::toupper((unsigned char)c);
    for (int a = 0; a < 20; ++a)
        if (ONE[a] == c) return a;
    return -1;
}

void atom_record(std::string& s, size_t serial, const char* name, int aa, char chain, size_t res_seq, float x, float y,
                 float z) {
    appendf(s, "ATOM  %5zu %-4s %-3s %c%4zu    %8.3f%8.3f%8.3f  1.00  0.00           C\n", serial, name, BT_AA3[aa],
            chain, res_seq, (double)x, (double)y, (double)z);
}

std::string json_escape(const char* p) {
    std::string o;
    for (; p && *p; ++p) {
        if (*p == '"') o += "\\\"";
        else if (*p == '\\') o += "\\\\";
        else if (*p == '\n') o += "\\n";
        else o += *p;
    }
    return o;
}

std::string csv_field(const char* p) {
    std::string o = "\"";
    for (; p && *p; ++p) {
        if (*p == '"') o += "\"\"";
        else o += *p;
    }
    return o + "\"";
}

}  // namespace

extern "C" {

int binder_parse_pdb_text(const char* text, size_t len, float* xyz, uint8_t* aa, size_t cap, size_t* out_n) {
    if (!out_n || (!text && len)) return BINDER_ERR_ARG;
    size_t n = 0, pos = 0;
    while (pos < len) {
        size_t eol = pos;
        while (eol < len && text[eol] != '\n') ++eol;
        std::string line(text + pos, eol - pos);
        if (!line.empty() && line.back() == '\r') line.pop_back();  // lines() drops a CR before the LF
        pos = eol + 1;
        if (line.compare(0, 4, "ATOM") != 0 && line.compare(0, 6, "HETATM") != 0) continue;
        std::string f;
        if (trim(field(line, 12, 16, f) ? f : "    ") != "CA") continue;
        const std::string res = trim(field(line, 17, 20, f) ? f : "   ");
        float c[3] = {0.f, 0.f, 0.f};
        for (int k = 0; k < 3; ++k) {
            float v;
            if (field(line, 30 + 8 * k, 38 + 8 * k, f) && parse_f32(trim(f), v)) c[k] = v;
        }
        if (n < cap) {
            if (xyz) {
                xyz[3 * n] = c[0];
                xyz[3 * n + 1] = c[1];
                xyz[3 * n + 2] = c[2];
            }
            if (aa) aa[n] = (uint8_t)aa_from_three(res);
        }
        ++n;
    }
    *out_n = n;
    if (n == 0) return BINDER_ERR_ARG;  // BinderError::EmptyInput
    return n > cap ? BINDER_ERR_CAPACITY : BINDER_OK;
}

int binder_parse_pdb_file(const char* path, float* xyz, uint8_t* aa, size_t cap, size_t* out_n) {
    if (!path || !out_n) return BINDER_ERR_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return BINDER_ERR_IO;
    std::string text;
    char buf[65536];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
    const bool bad = std::ferror(f) != 0;
    std::fclose(f);
    if (bad) return BINDER_ERR_IO;
    return binder_parse_pdb_text(text.data(), text.size(), xyz, aa, cap, out_n);
}

int binder_parse_peptide(const char* seq, float* xyz, uint8_t* aa, size_t cap, size_t* out_n) {
    if (!seq || !out_n) return BINDER_ERR_ARG;
    const size_t n = std::strlen(seq);
    *out_n = n;
    if (n == 0) return BINDER_ERR_ARG;  // BinderError::EmptyInput
    for (size_t i = 0; i < n; ++i)
        if (aa_from_one(seq[i]) < 0) return BINDER_ERR_ARG;  // unknown one-letter code
    if (n > cap) return BINDER_ERR_CAPACITY;
    for (size_t i = 0; i < n; ++i) {
        if (xyz) {
            xyz[3 * i] = ((float)i - (float)n * 0.5f) * 3.8f;
            xyz[3 * i + 1] = 0.0f;
            xyz[3 * i + 2] = 0.0f;
        }
        if (aa) aa[i] = (uint8_t)aa_from_one(seq[i]);
    }
    return BINDER_OK;
}

int binder_write_pdb_ca(size_t n, const float* xyz, const uint8_t* aa, char chain, char* out, size_t cap,
                        size_t* out_len) {
    if (n && (!xyz || !aa)) return BINDER_ERR_ARG;
    std::string s;
    s.reserve(n * 81 + 4);
    for (size_t i = 0; i < n; ++i) {
        if (aa[i] >= 20) return BINDER_ERR_ARG;
        atom_record(s, std::min<size_t>(i + 1, 99999), " CA ", aa[i], chain, std::min<size_t>(i + 1, 9999),
                    xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    }
    s += "END\n";
    return emit(s, out, cap, out_len);
}

int binder_write_pdb_multi(size_t n_chains, const size_t* n_res, const uint8_t* aa, const float* pos,
                           const char* chain_ids, char* out, size_t cap, size_t* out_len) {
    if (n_chains && (!n_res || !chain_ids)) return BINDER_ERR_ARG;
    std::string s;
    size_t serial = 0, r0 = 0;
    for (size_t c = 0; c < n_chains; ++c) {
        if (n_res[c] && (!aa || !pos)) return BINDER_ERR_ARG;
        for (size_t r = 0; r < n_res[c]; ++r) {
            const int a = aa[r0 + r];
            if (a >= 20) return BINDER_ERR_ARG;
            for (int k = 0; k < BT_TOPO_N[a]; ++k) {
                ++serial;
                const float* p = pos + ((r0 + r) * BINDER_MAX_SLOTS + k) * 3;
                atom_record(s, std::min<size_t>(serial, 99999), BT_SLOT_NAME[a][k], a, chain_ids[c],
                            std::min<size_t>(r + 1, 9999), p[0], p[1], p[2]);
            }
        }
        r0 += n_res[c];
        s += "TER\n";
    }
    s += "END\n";
    return emit(s, out, cap, out_len);
}

int binder_write_pdb_allatom(size_t n_res, const uint8_t* aa, const float* pos, char chain, char* out, size_t cap,
                             size_t* out_len) {
    if (n_res && (!aa || !pos)) return BINDER_ERR_ARG;
    std::string s;
    size_t serial = 0;
    for (size_t r = 0; r < n_res; ++r) {
        const int a = aa[r];
        if (a >= 20) return BINDER_ERR_ARG;
        for (int k = 0; k < BT_TOPO_N[a]; ++k) {
            ++serial;
            const float* p = pos + (r * BINDER_MAX_SLOTS + k) * 3;
            atom_record(s, std::min<size_t>(serial, 99999), BT_SLOT_NAME[a][k], a, chain, std::min<size_t>(r + 1, 9999),
                        p[0], p[1], p[2]);
        }
    }
    s += "END\n";
    return emit(s, out, cap, out_len);
}

int binder_write_fasta(const binder_candidate_report* rep, size_t n, char* out, size_t cap, size_t* out_len) {
    if (n && !rep) return BINDER_ERR_ARG;
    std::string s;
    for (size_t i = 0; i < n; ++i) {
        const binder_candidate_report& r = rep[i];
        const char* seq = r.sequence ? r.sequence : "";
        if (r.light_sequence) {
            appendf(s, ">candidate_%d_VH E=%.4f\n", r.rank, (double)r.energy);
            s += seq;
            s += "\n";
            appendf(s, ">candidate_%d_VL E=%.4f\n", r.rank, (double)r.energy);
            s += r.light_sequence;
            s += "\n";
        } else {
            appendf(s, ">candidate_%d E=%.4f\n", r.rank, (double)r.energy);
            s += seq;
            s += "\n";
        }
    }
    return emit(s, out, cap, out_len);
}

int binder_write_json(const binder_candidate_report* rep, size_t n, char* out, size_t cap, size_t* out_len) {
    if (n && !rep) return BINDER_ERR_ARG;
    std::string s = "[\n";
    for (size_t i = 0; i < n; ++i) {
        const binder_candidate_report& r = rep[i];
        s += "  {\n";
        appendf(s, "    \"rank\": %d,\n", r.rank);
        s += "    \"sequence\": \"" + json_escape(r.sequence) + "\",\n";
        if (r.light_sequence) s += "    \"light_sequence\": \"" + json_escape(r.light_sequence) + "\",\n";
        else s += "    \"light_sequence\": null,\n";
        appendf(s, "    \"energy\": %.6f,\n", (double)r.energy);
        appendf(s, "    \"entropy_penalty\": %.6f,\n", (double)r.entropy_penalty);
        appendf(s, "    \"dg_corrected\": %.6f,\n", (double)r.dg_corrected);
        appendf(s, "    \"net_charge\": %d,\n", r.net_charge);
        appendf(s, "    \"aggregation_risk\": %s,\n", r.aggregation_risk ? "true" : "false");
        appendf(s, "    \"n_interface\": %d,\n", r.n_interface);
        if (r.clashes >= 0) appendf(s, "    \"clashes\": %d,\n", r.clashes);
        else s += "    \"clashes\": null,\n";
        if (r.rama_outliers >= 0) appendf(s, "    \"rama_outliers\": %d\n", r.rama_outliers);
        else s += "    \"rama_outliers\": null\n";
        s += i + 1 < n ? "  },\n" : "  }\n";
    }
    s += "]\n";
    return emit(s, out, cap, out_len);
}

int binder_write_csv(const binder_candidate_report* rep, size_t n, char* out, size_t cap, size_t* out_len) {
    if (n && !rep) return BINDER_ERR_ARG;
    std::string s =
        "rank,sequence,light_sequence,energy,entropy_penalty,dg_corrected,net_charge,aggregation_risk,n_interface,"
        "clashes,rama_outliers\n";
    for (size_t i = 0; i < n; ++i) {
        const binder_candidate_report& r = rep[i];
        appendf(s, "%d,", r.rank);
        s += csv_field(r.sequence) + "," + csv_field(r.light_sequence ? r.light_sequence : "") + ",";
        appendf(s, "%.6f,%.6f,%.6f,%d,%s,%d,", (double)r.energy, (double)r.entropy_penalty, (double)r.dg_corrected,
                r.net_charge, r.aggregation_risk ? "true" : "false", r.n_interface);
        if (r.clashes >= 0) appendf(s, "%d", r.clashes);
        s += ",";
        if (r.rama_outliers >= 0) appendf(s, "%d", r.rama_outliers);
        s += "\n";
    }
    return emit(s, out, cap, out_len);
}

}  // extern "C"
