/*
 * Stand-in for the reference's FPGA configuration class (which needs the
 * hybridsys FPGA layer and the ADM-XRC3 driver headers), used ONLY to compile
 * the reference's VCFData.cpp into the writer harness of the test oracle.
 * The harness passes no FPGA configuration; these getters are never called.
 */
#ifndef FPGACONFIGURATIONEAGLEIMP_H_
#define FPGACONFIGURATIONEAGLEIMP_H_

#include <cstddef>
#include <cstdint>

class FPGAConfigurationEagleImp {
public:
    uint64_t getAvailableRAM() const { return 0; }
    unsigned getNumPipelines() const { return 0; }
    size_t getMaxSites() const { return 0; }
    size_t getMaxHaps() const { return 0; }
    size_t getMaxK() const { return 0; }
};

#endif
