// Winner artefacts (model_artifact/winner_artifact.hpp:12-36, winner_artifact.cpp:13-188 and :218-280,
// winner_artifact_reader.cpp:12-247): the best individual's genome image as a .bin file and its metadata as a
// JSON file (format_version 2: timestamp, generation, fitness, indices, action count, byte count, seed, the
// action-space path and the first action_count catalog words as upper-case ASCII), each written to path.tmp and
// renamed. The reader follows the reference's: each key is found by its first quoted occurrence, numbers are the
// maximal run of number characters after the colon, the word list must hold action_count five-letter upper-case
// words, and the .bin must hold exactly genome_byte_count bytes. Host code only.
#include <charconv>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iterator>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/nwg_capi.h"
#include "nwg_internal.cuh"

using namespace nwg;

namespace {

constexpr int kFormatVersion = 2;

std::string EscapeJson(const std::string &in) {
    std::string out;
    out.reserve(in.size());
    for (const char c : in) {
        switch (c) {
        case '\\': out += "\\\\"; break;
        case '"': out += "\\\""; break;
        case '\n': out += "\\n"; break;
        case '\r': out += "\\r"; break;
        case '\t': out += "\\t"; break;
        default: out += c; break;
        }
    }
    return out;
}

std::string LocalTimestamp() {
    const std::time_t now = std::time(nullptr);
    std::tm local{};
    if (localtime_r(&now, &local) == nullptr) {
        return std::string();
    }
    char text[32];
    return std::strftime(text, sizeof(text), "%Y-%m-%dT%H:%M:%S", &local) > 0 ? std::string(text) : std::string();
}

bool ValidLetters(const std::uint8_t *letters, std::size_t count) {
    for (std::size_t i = 0; i < count * 5; ++i) {
        if (letters[i] >= 26) {
            return false;
        }
    }
    return true;
}

// The metadata document, formatted as the reference's stream writes it (default float formatting).
std::string MetadataJson(const nwg_winner_metadata &m, const std::uint8_t *letters, const std::string &path,
                         const std::string &timestamp) {
    std::ostringstream s;
    s << "{\n"
      << "  \"format_version\": " << kFormatVersion << ",\n"
      << "  \"timestamp_local\": \"" << EscapeJson(timestamp) << "\",\n"
      << "  \"generation_index\": " << m.generation_index << ",\n"
      << "  \"best_fitness\": " << m.best_fitness << ",\n"
      << "  \"best_index\": " << m.best_index << ",\n"
      << "  \"best_slot_index\": " << m.best_slot_index << ",\n"
      << "  \"action_count\": " << m.action_count << ",\n"
      << "  \"genome_byte_count\": " << m.genome_byte_count << ",\n"
      << "  \"seed\": " << m.seed << ",\n"
      << "  \"action_space_path\": \"" << EscapeJson(path) << "\",\n"
      << "  \"action_space_words\": [";
    for (std::size_t w = 0; w < m.action_count; ++w) {
        if (w != 0) {
            s << ", ";
        }
        s << '"';
        for (std::size_t k = 0; k < 5; ++k) {
            s << static_cast<char>('A' + letters[w * 5 + k]);
        }
        s << '"';
    }
    s << "]\n}\n";
    return s.str();
}

bool WriteFile(const std::string &path, const void *data, std::size_t n) {
    std::FILE *f = std::fopen(path.c_str(), "wb");
    if (f == nullptr) {
        return false;
    }
    const bool ok = std::fwrite(data, 1, n, f) == n;
    return std::fclose(f) == 0 && ok;
}

bool ReadFile(const std::string &path, std::string &out) {
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) {
        return false;
    }
    out.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
    return in.good() || in.eof();
}

bool IsSpace(char c) { return c == ' ' || c == '\n' || c == '\r' || c == '\t'; }

bool Locate(const std::string &json, const char *key, std::size_t &pos) {
    const std::string needle = std::string("\"") + key + "\"";
    const std::size_t k = json.find(needle);
    if (k == std::string::npos) {
        return false;
    }
    const std::size_t colon = json.find(':', k + needle.size());
    if (colon == std::string::npos) {
        return false;
    }
    pos = colon + 1;
    while (pos < json.size() && IsSpace(json[pos])) {
        ++pos;
    }
    return pos < json.size();
}

bool ReadString(const std::string &json, const char *key, std::string &out) {
    std::size_t p = 0;
    if (!Locate(json, key, p) || json[p] != '"') {
        return false;
    }
    out.clear();
    for (++p; p < json.size(); ++p) {
        const char c = json[p];
        if (c == '"') {
            return true;
        }
        if (c != '\\') {
            out += c;
            continue;
        }
        if (++p >= json.size()) {
            return false;
        }
        switch (json[p]) {
        case '\\':
        case '"': out += json[p]; break;
        case 'n': out += '\n'; break;
        case 'r': out += '\r'; break;
        case 't': out += '\t'; break;
        default: return false;
        }
    }
    return false;
}

template <typename T>
bool ReadNumber(const std::string &json, const char *key, T &out) {
    std::size_t p = 0;
    if (!Locate(json, key, p)) {
        return false;
    }
    const char *begin = json.data() + p;
    const char *end = begin;
    const char *stop = json.data() + json.size();
    while (end < stop && (*end == '-' || *end == '+' || *end == '.' || (*end >= '0' && *end <= '9') || *end == 'e' ||
                          *end == 'E')) {
        ++end;
    }
    return begin != end && std::from_chars(begin, end, out).ec == std::errc{};
}

bool ReadWords(const std::string &json, const char *key, std::vector<std::uint8_t> &letters) {
    std::size_t p = 0;
    if (!Locate(json, key, p) || json[p] != '[') {
        return false;
    }
    letters.clear();
    for (++p; p < json.size();) {
        while (p < json.size() && (IsSpace(json[p]) || json[p] == ',')) {
            ++p;
        }
        if (p >= json.size()) {
            return false;
        }
        if (json[p] == ']') {
            return !letters.empty();
        }
        if (json[p] != '"' || letters.size() / 5 >= NWG_CATALOG_CAPACITY) {
            return false;
        }
        std::string word;
        for (++p; p < json.size() && json[p] != '"'; ++p) {
            word += json[p];
        }
        if (p >= json.size() || word.size() != 5) {
            return false;
        }
        ++p;
        for (const char c : word) {
            if (c < 'A' || c > 'Z') {
                return false;
            }
            letters.push_back(static_cast<std::uint8_t>(c - 'A'));
        }
    }
    return false;
}

bool CopyOut(const std::string &text, char *out, std::size_t capacity) {
    if (out == nullptr) {
        return true;
    }
    if (text.size() + 1 > capacity) {
        return false;
    }
    std::memcpy(out, text.c_str(), text.size() + 1);
    return true;
}

}  // namespace

extern "C" {

int nwg_winner_artifact_write(const char *binary_path, const char *metadata_path, const uint8_t *genome_bytes,
                              const nwg_winner_metadata *metadata, const uint8_t *catalog_letters,
                              size_t catalog_count, const char *action_space_path, const char *timestamp_local) {
    // IsValidWinnerArtifactInputs (winner_artifact.cpp:13-18) and the path checks of the paths variant
    if (binary_path == nullptr || metadata_path == nullptr || genome_bytes == nullptr || metadata == nullptr ||
        catalog_letters == nullptr || metadata->action_count == 0 || metadata->genome_byte_count == 0 ||
        catalog_count > NWG_CATALOG_CAPACITY || metadata->action_count > catalog_count ||
        !ValidLetters(catalog_letters, catalog_count) || std::strcmp(binary_path, metadata_path) == 0 ||
        binary_path[0] == '\0' || metadata_path[0] == '\0') {
        return kInvalidRuntimeConfig;
    }
    const std::string timestamp = timestamp_local != nullptr ? std::string(timestamp_local) : LocalTimestamp();
    const std::string json = MetadataJson(*metadata, catalog_letters,
                                          action_space_path != nullptr ? action_space_path : "", timestamp);
    const std::string bin_tmp = std::string(binary_path) + ".tmp";
    const std::string json_tmp = std::string(metadata_path) + ".tmp";
    const bool ok = WriteFile(bin_tmp, genome_bytes, metadata->genome_byte_count) &&
                    WriteFile(json_tmp, json.data(), json.size()) && std::rename(bin_tmp.c_str(), binary_path) == 0 &&
                    std::rename(json_tmp.c_str(), metadata_path) == 0;
    if (!ok) {
        std::remove(bin_tmp.c_str());
        std::remove(json_tmp.c_str());
        return kInvalidRuntimeConfig;
    }
    return kOk;
}

int nwg_winner_artifact_persist(const nwg_runtime *rt, uint32_t seed, const uint8_t *catalog_letters,
                                size_t catalog_count, const char *action_space_path, const char *binary_path,
                                const char *metadata_path, const char *timestamp_local) {
    nwg_fitness_summary summary{};
    int st = nwg_read_summary(rt, &summary);
    if (st != kOk) {
        return st;
    }
    nwg_runtime_info info{};
    st = nwg_get_info(rt, &info);
    if (st != kOk) {
        return st;
    }
    std::vector<std::uint8_t> genome(info.slot_stride_bytes);
    std::size_t got = 0;
    st = nwg_download_slot(rt, summary.best_slot_index, genome.data(), genome.size(), &got);
    if (st != kOk) {
        return st;
    }
    // MakeWinnerArtifactMetadata (cli/run_genetic_algorithm.cu:1504-1517)
    nwg_winner_metadata m{};
    m.best_fitness = summary.best_fitness;
    m.generation_index = summary.generation_index;
    m.best_index = summary.best_index;
    m.best_slot_index = summary.best_slot_index;
    m.action_count = summary.action_count;
    m.genome_byte_count = got;
    m.seed = seed;
    return nwg_winner_artifact_write(binary_path, metadata_path, genome.data(), &m, catalog_letters, catalog_count,
                                     action_space_path, timestamp_local);
}

int nwg_winner_artifact_read(const char *binary_path, const char *metadata_path, nwg_winner_metadata *metadata,
                             uint8_t *genome_bytes, size_t genome_capacity, uint8_t *catalog_letters,
                             size_t *catalog_count, char *action_space_path, size_t path_capacity,
                             char *timestamp_local, size_t timestamp_capacity) {
    if (binary_path == nullptr || metadata_path == nullptr || metadata == nullptr) {
        return kInvalidRuntimeConfig;
    }
    std::memset(metadata, 0, sizeof(*metadata));
    std::string json, binary, path, timestamp;
    std::size_t version = 0;
    nwg_winner_metadata m{};
    std::vector<std::uint8_t> letters;
    const bool ok = ReadFile(metadata_path, json) && ReadNumber(json, "format_version", version) &&
                    static_cast<int>(version) == kFormatVersion && ReadString(json, "timestamp_local", timestamp) &&
                    ReadNumber(json, "generation_index", m.generation_index) &&
                    ReadNumber(json, "best_fitness", m.best_fitness) && ReadNumber(json, "best_index", m.best_index) &&
                    ReadNumber(json, "best_slot_index", m.best_slot_index) &&
                    ReadNumber(json, "action_count", m.action_count) &&
                    ReadNumber(json, "genome_byte_count", m.genome_byte_count) && ReadNumber(json, "seed", m.seed) &&
                    ReadString(json, "action_space_path", path) && ReadWords(json, "action_space_words", letters) &&
                    ReadFile(binary_path, binary) && !binary.empty() && binary.size() == m.genome_byte_count &&
                    m.action_count == letters.size() / 5 && m.action_count > 0;
    if (!ok) {
        return kInvalidRuntimeConfig;
    }
    if ((genome_bytes != nullptr && genome_capacity < binary.size()) ||
        !CopyOut(path, action_space_path, path_capacity) || !CopyOut(timestamp, timestamp_local, timestamp_capacity)) {
        return kInvalidRuntimeConfig;
    }
    if (genome_bytes != nullptr) {
        std::memcpy(genome_bytes, binary.data(), binary.size());
    }
    if (catalog_letters != nullptr) {
        std::memcpy(catalog_letters, letters.data(), letters.size());
    }
    if (catalog_count != nullptr) {
        *catalog_count = letters.size() / 5;
    }
    *metadata = m;
    return kOk;
}

}  // extern "C"
