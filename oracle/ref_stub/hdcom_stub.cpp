// Link-time stand-ins for the four hdcom::HdCommunication methods that the
// reference CPU filter and noise sources reference
// (Denoiser/iternlm_cpu.cpp:73,81,551-552; Noise/noiselevel.cpp:308).
// They are reached only in --resume and disk-block modes, which the oracle
// never enables; reaching one is a harness bug, so each aborts.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include "Geometry/hdcommunication.h"

namespace hdcom {
static void oracle_io_unreachable(const char* what) {
    std::fprintf(stderr, "oracle: reference IO path reached (%s); not supported\n", what);
    std::abort();
}
std::vector<std::string> HdCommunication::GetFilelist(std::string, int*) {
    oracle_io_unreachable("GetFilelist");
    return {};
}
float* HdCommunication::Get3DTifSequence_32bitPointer(std::vector<std::string>&, int*, int, int) {
    oracle_io_unreachable("Get3DTifSequence_32bitPointer");
    return nullptr;
}
void HdCommunication::SaveTifSequence_32bit(int, float*, int*, std::string, std::string, bool) {
    oracle_io_unreachable("SaveTifSequence_32bit");
}
void HdCommunication::SaveTifSequence_as16bit(int, float*, int*, std::string, std::string, bool) {
    oracle_io_unreachable("SaveTifSequence_as16bit");
}
}  // namespace hdcom
