// Reference checkpoint formats: the reference's own host I/O of the particle path
// (inc/swarm/swarm_host.cuh: save_host_binary / load_host_binary :778-815, save_sam_as_velocity
// :864-880, load_velocity_as_sam :883-899, frame_num :906-913), compiled from the GameDev tree
// where it lies against a generated model header, by oracle/ref/Makefile into
// oracle/_ref/io_<model>_<n>/ref_io.  TEST INFRASTRUCTURE ONLY: it pins the library's checkpoint
// writer and reader (gd_save_checkpoint, gd_load_checkpoint) byte for byte.
//
//   ref_io save  <in.bin> <out.dat>   in.bin: int32 n (= N_P), then n records in the internal
//                                     (angular-velocity) layout; out.dat: the particle file the
//                                     reference writes for them (SAVE_PARTICLE_TO_FILE)
//   ref_io load  <in.dat> <out.bin>   a particle file read as LOAD_PARTICLE_TO_VRAM reads it
//                                     (size-checked), back in the internal layout, int32 n first
//   ref_io frame <idx>                prints frame_num(idx)
//   ref_io variables <out.txt> <total_dust_mass>
//                                     the run's parameter file as save_variable writes it
//                                     (swarm_host.cuh:989-1143)
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include <swarm_host.cuh>

int main(int argc, char **argv) {
    if (argc == 3 && std::string(argv[1]) == "frame") {
        std::printf("%s\n", frame_num(std::atoi(argv[2])).c_str());
        return 0;
    }
    if (argc == 4 && std::string(argv[1]) == "variables")
        return save_variable(argv[2], std::strtod(argv[3], nullptr)) ? 0 : 4;
    if (argc != 4) {
        std::fprintf(stderr, "usage: ref_io save|load <in> <out> | ref_io frame <idx> | ref_io variables <out> <mass>\n");
        return 2;
    }
    const std::string mode = argv[1];
    std::vector<swarm> particle(N_P);
    if (mode == "save") {
        std::ifstream in(argv[2], std::ios::binary);
        int n = 0;
        in.read(reinterpret_cast<char *>(&n), 4);
        if (!in || n != N_P) return 3;
        in.read(reinterpret_cast<char *>(particle.data()), sizeof(swarm) * N_P);
        if (!in) return 3;
        save_sam_as_velocity(particle.data());
        return save_host_binary(argv[3], particle.data(), N_P) ? 0 : 4;
    }
    if (mode == "load") {
        if (!load_host_binary(argv[2], particle.data(), N_P)) return 5;
        load_velocity_as_sam(particle.data());
        std::ofstream out(argv[3], std::ios::binary);
        const int n = N_P;
        out.write(reinterpret_cast<const char *>(&n), 4);
        out.write(reinterpret_cast<const char *>(particle.data()), sizeof(swarm) * N_P);
        return out ? 0 : 4;
    }
    return 2;
}
