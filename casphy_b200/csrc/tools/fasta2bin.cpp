// Drop-in for `fasta2bin <input FASTA file> <output prefix>` (cu/fasta2bin.cu:
// 245-363): <prefix>.bin ({nseq, enc_len} + encoded variable columns),
// <prefix>_names.txt ("SequenceName,ValidBaseCount") and
// <prefix>_positions.txt ("Position,IsVariable").  The FASTA text is read on
// the host with the reference's rules (:120-183): a header line starts with
// '>', the name is its first token, whitespace inside sequence lines is
// dropped, blank lines are skipped, a header without sequence lines is
// dropped; the columns are classified and encoded on the GPU.
//
// The process is one-shot, so CUDA start-up is most of its time: a second
// thread selects the device (creating its context) while this one reads the
// file.  The text is read in one piece and the sequence letters go straight
// into the row-major matrix that the encoder takes.
#include <cstdio>
#include <cstring>
#include <iostream>
#include <fstream>
#include <string>
#include <thread>
#include <vector>

#include "casphy.h"
#include "toolio.h"

namespace {

struct Record {
    std::string name;
    size_t begin, end;  // letters [begin, end) of the matrix
    int valid;          // letters other than '-', '.', 'N', 'n' (cu/fasta2bin.cu:168-175)
};

// False only when the file does not open; a read error ends the text where it
// happened, as it ends std::getline's lines.
bool read_all(const char* path, std::vector<char>& text) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    size_t n = 0;
    text.resize(size_t(1) << 24);
    for (;;) {
        n += std::fread(text.data() + n, 1, text.size() - n, f);
        if (n < text.size()) break;
        text.resize(text.size() * 2);
    }
    std::fclose(f);
    text.resize(n);
    return true;
}

// Lines split at '\n' as std::getline does (a last line without one counts).
void parse(const std::vector<char>& text, std::vector<char>& mat, std::vector<Record>& recs) {
    bool space[256] = {}, invalid[256] = {};
    for (unsigned char c : {' ', '\t', '\n', '\v', '\f', '\r'}) space[c] = true;
    for (unsigned char c : {'-', '.', 'N', 'n'}) invalid[c] = true;
    mat.resize(text.size());
    char* out = mat.data();
    size_t nOut = 0, seqBegin = 0;
    int valid = 0;
    std::string name;
    auto flush = [&]() {
        if (nOut > seqBegin) recs.push_back({name, seqBegin, nOut, valid});
        seqBegin = nOut;
        valid = 0;
    };
    const char* p = text.data();
    const char* const end = p + text.size();
    while (p < end) {
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
        const char* le = nl ? nl : end;
        if (le > p) {
            if (*p == '>') {
                flush();
                name.assign(p + 1, le);
                const size_t fns = name.find_first_not_of(" \t"), fs = name.find_first_of(" \t");
                if (fns != std::string::npos) name = fs != std::string::npos ? name.substr(fns, fs - fns) : name.substr(fns);
            } else {
                for (const char* q = p; q < le; q++) {
                    const unsigned char c = (unsigned char)*q;
                    if (space[c]) continue;
                    out[nOut++] = (char)c;
                    valid += !invalid[c];
                }
            }
        }
        p = nl ? nl + 1 : end;
    }
    flush();
    mat.resize(nOut);
}

}  // namespace

int main(int argc, char* argv[]) {
    if (argc != 3) {
        std::cout << "Usage: " << argv[0] << " <input FASTA file> <output prefix>" << std::endl;
        return 1;
    }
    const std::string prefix = argv[2];
    int dev = -1;
    std::string devError;
    std::thread starter([&]() {
        dev = tool::pick_device();
        if (dev < 0) devError = casphy_last_error();
    });
    std::vector<char> text, mat;
    std::vector<Record> recs;
    const bool opened = read_all(argv[1], text);
    if (opened) parse(text, mat, recs);
    std::vector<char>().swap(text);
    starter.join();
    if (!opened) {
        std::cerr << "Error: Cannot open file: " << argv[1] << std::endl;
        return 1;
    }
    if (recs.empty()) {
        std::cerr << "Error: No valid sequences found in file" << std::endl;
        return 1;
    }
    const size_t len = recs[0].end - recs[0].begin;
    for (const auto& r : recs)
        if (r.end - r.begin != len) {
            std::cerr << "Error: All sequences must have the same length for variant filtering" << std::endl;
            return 1;
        }
    if (dev < 0 || casphy_set_device(dev) != CASPHY_OK) {  // the current device is per thread
        fprintf(stderr, "fasta2bin: %s (%s)\n", casphy_strerror(CASPHY_ENODEV),
                dev < 0 ? devError.c_str() : casphy_last_error());
        return 1;
    }
    std::vector<uint8_t> var(len);
    uint32_t nkeep = 0;
    const uint32_t nseq = (uint32_t)recs.size();
    std::vector<uint32_t> bin((size_t)nseq * ((len + 3) / 4) + 1);
    const int rc = casphy_fasta_encode(nseq, (uint32_t)len, mat.data(), var.data(), &nkeep, bin.data(), bin.size());
    if (rc) return tool::fail("fasta2bin", rc);
    std::cout << "Found " << nseq << " sequences" << std::endl;
    std::cout << "Removed " << (len - nkeep) << " non-variable positions" << std::endl;
    {
        std::ofstream out(prefix + "_positions.txt");
        out << "Position,IsVariable\n";
        for (size_t i = 0; i < len; i++) out << i << "," << (var[i] ? "Yes" : "No") << "\n";
    }
    {
        std::ofstream out(prefix + "_names.txt");
        out << "SequenceName,ValidBaseCount\n";
        for (const auto& r : recs) out << r.name << "," << r.valid << '\n';
    }
    {
        std::ofstream out(prefix + ".bin", std::ios::binary);
        const uint32_t hdr[2] = {nseq, (nkeep + 3) / 4};
        out.write(reinterpret_cast<const char*>(hdr), sizeof(hdr));
        out.write(reinterpret_cast<const char*>(bin.data()), sizeof(uint32_t) * (size_t)nseq * hdr[1]);
    }
    std::cout << "Conversion completed!" << std::endl;
    return 0;
}
