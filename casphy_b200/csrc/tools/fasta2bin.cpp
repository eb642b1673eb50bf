// Drop-in for `fasta2bin <input FASTA file> <output prefix>` (cu/fasta2bin.cu:
// 245-363): <prefix>.bin ({nseq, enc_len} + encoded variable columns),
// <prefix>_names.txt ("SequenceName,ValidBaseCount") and
// <prefix>_positions.txt ("Position,IsVariable").  The FASTA text is read on
// the host with the reference's rules (:120-183): a header line starts with
// '>', the name is its first token, whitespace inside sequence lines is
// dropped, blank lines are skipped, a header without sequence lines is
// dropped; the columns are classified and encoded on the GPU.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "casphy.h"
#include "toolio.h"

static int valid_bases(const std::string& s) {
    int n = 0;
    for (char c : s) {
        const char u = (char)std::toupper((unsigned char)c);
        if (u != '-' && u != '.' && u != 'N') n++;
    }
    return n;
}

int main(int argc, char* argv[]) {
    if (argc != 3) {
        std::cout << "Usage: " << argv[0] << " <input FASTA file> <output prefix>" << std::endl;
        return 1;
    }
    const std::string prefix = argv[2];
    std::vector<std::string> names, seqs;
    std::vector<int> valid;
    {
        std::ifstream file(argv[1]);
        if (!file.is_open()) {
            std::cerr << "Error: Cannot open file: " << argv[1] << std::endl;
            return 1;
        }
        std::string name, seq, line;
        auto flush = [&]() {
            if (!seq.empty()) {
                seqs.push_back(seq);
                names.push_back(name);
                valid.push_back(valid_bases(seq));
                seq.clear();
            }
        };
        while (std::getline(file, line)) {
            if (line.empty()) continue;
            if (line[0] == '>') {
                flush();
                name = line.substr(1);
                const size_t fns = name.find_first_not_of(" \t"), fs = name.find_first_of(" \t");
                if (fns != std::string::npos) name = fs != std::string::npos ? name.substr(fns, fs - fns) : name.substr(fns);
            } else {
                line.erase(std::remove_if(line.begin(), line.end(), [](unsigned char c) { return std::isspace(c); }),
                           line.end());
                seq += line;
            }
        }
        flush();
    }
    if (seqs.empty()) {
        std::cerr << "Error: No valid sequences found in file" << std::endl;
        return 1;
    }
    const size_t len = seqs[0].size();
    for (const auto& s : seqs)
        if (s.size() != len) {
            std::cerr << "Error: All sequences must have the same length for variant filtering" << std::endl;
            return 1;
        }
    const int dev = tool::pick_device();
    if (dev < 0) return tool::fail("fasta2bin", CASPHY_ENODEV);
    std::vector<char> mat(seqs.size() * len);
    for (size_t i = 0; i < seqs.size(); i++) std::copy(seqs[i].begin(), seqs[i].end(), mat.begin() + i * len);
    std::vector<uint8_t> var(len);
    uint32_t nkeep = 0;
    const uint32_t nseq = (uint32_t)seqs.size();
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
        for (size_t i = 0; i < names.size(); i++) out << names[i] << "," << valid[i] << '\n';
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
