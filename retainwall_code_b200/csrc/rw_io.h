// Case files and output files in the reference's layouts (src/loquat_io.cu).
#pragma once
#include <map>
#include <string>
#include <vector>

#include "../../include/retainwall.h"

namespace rw {

// Host copy of a case as read from <project>.xml/.dat/.motion.
struct HostCase {
  rw_case_params params{};
  std::vector<int32_t> codes;
  std::vector<double> pospres, velrhop, idmassidx, stress, strain, normal;
  rw_case view() const;  // rw_case pointing into this object
};

// LoquatIo::LoadParameters + LoadParticles (src/loquat_io.cu:75-312).
// Returns RW_OK or an error code with a message in *msg.
int read_project(const std::string& project, HostCase* out, std::string* msg);
// Typed parameter map of an XML parameter file (tag -> (type, text)).
int read_xml_params(const std::string& path, std::map<std::string, std::pair<std::string, std::string>>* out,
                    std::string* msg);

// Arrays of one output frame, reference row layouts, double precision.
struct Frame {
  int np = 0, npb = 0, npm = 0;
  std::vector<int32_t> codes;       // np x 4
  std::vector<double> pos, vel, acc, idm, normal;  // np x 4 (normal: npb x 4)
  std::vector<double> str, stn;     // np x 6
};

// LoquatIo::SaveXml (src/loquat_io.cu:315-399).
int write_output_xml(const std::string& path, const rw_case_params& p, int np, int npb, int npm, double time,
                     double dt, int output_number);
// LoquatIo::SaveParticles format 1 (src/loquat_io.cu:430-468).
int write_frame_dat(const std::string& path, const Frame& f);
// LoquatIo::SaveParticles format 2 (src/loquat_io.cu:470-680): one <id>_<n>.vtu per block id.
int write_frame_vtu(const std::string& dir, int output_number, const Frame& f);

// SaveDatFile layout of a case (src/GenCase.cu:70-116).
int write_case_dat(const rw_case* c, const std::string& path);

}  // namespace rw
