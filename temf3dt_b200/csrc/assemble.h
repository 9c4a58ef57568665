#pragma once
#include "ctx.h"

namespace temf {
void build_adjacency(const temf_ctx& c, std::vector<int64_t>& xadj, std::vector<int>& adj);
void build_pattern(const temf_ctx& c, const std::vector<int>& perm, const std::vector<int>& iperm, Pattern& P);
void upload_mesh(temf_ctx& c);
void upload_media(temf_ctx& c);
void upload_pattern(temf_ctx& c);
void launch_assembly(temf_ctx& c);
// bit f of mask[t] set when local face f of tet t lies on the mesh boundary
void boundary_face_mask(const temf_ctx& c, std::vector<unsigned char>& mask);
}  // namespace temf
