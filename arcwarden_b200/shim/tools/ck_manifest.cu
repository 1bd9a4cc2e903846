// ck_manifest — print a checkpoint file's header and manifest as the
// reference's own reader sees them (arc::checkpoint_read_header,
// include/pic/checkpoint.hpp:103-135): "seed S step N deck D git G", then
// "name dtype count" per array. Used to check that the files libarcb200 writes
// (aw_checkpoint_write) are read by the reference.
#include "pic/checkpoint.hpp"

#include <cstdio>
#include <exception>

int main(int argc, char** argv) {
    if (argc != 2) {
        std::fprintf(stderr, "usage: %s <checkpoint file>\n", argv[0]);
        return 2;
    }
    try {
        const arc::CheckpointHeader h = arc::checkpoint_read_header(argv[1]);
        std::printf("seed %llu step %lld deck %s git %s\n", static_cast<unsigned long long>(h.rng_seed),
                    static_cast<long long>(h.step), h.deck.c_str(), h.git_hash.c_str());
        for (const auto& a : h.manifest)
            std::printf("%s %u %llu\n", a.name.c_str(), a.dtype, static_cast<unsigned long long>(a.count));
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
