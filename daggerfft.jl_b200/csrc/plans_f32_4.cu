// Generated by gen_plans.py -- do not edit.
#include "static_plans.h"
namespace dfft {
template __global__ void axis_pass_static<float,true,1024,5,1,5>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,5,1,5>(const PassDesc);
template __global__ void axis_pass_static<float,true,1024,15,1,15>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,15,1,15>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,15,1,15>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,15,1,15>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,27,9,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,27,9,3,3,3>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,27,9,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,27,9,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,48,6,6,8>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,48,6,6,8>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,48,6,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,48,6,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,75,5,15,5>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,75,5,15,5>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,75,5,15,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,75,5,15,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,108,18,6,6,3>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,108,18,6,6,3>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,108,18,6,6,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,108,18,6,6,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,512,150,10,15,10>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,150,10,15,10>(const PassDesc);
template __global__ void axis_pass_pipe<float,512,false,16,150,10,15,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,512,true,0,150,10,15,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,216,36,6,6,6>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,216,36,6,6,6>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,216,36,6,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,216,36,6,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,512,270,18,15,6,3>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,270,18,15,6,3>(const PassDesc);
template __global__ void axis_pass_pipe<float,512,false,16,270,18,15,6,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,512,true,0,270,18,15,6,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,375,25,15,5,5>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,375,25,15,5,5>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,375,25,15,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,375,25,15,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,480,48,10,6,8>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,480,48,10,6,8>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,480,48,10,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,480,48,10,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,600,60,10,10,6>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,600,60,10,10,6>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,600,60,10,10,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,600,60,10,10,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,729,243,3,3,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,729,243,3,3,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,4,729,243,3,3,3,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,729,243,3,3,3,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,512,900,60,15,10,6>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,900,60,15,10,6>(const PassDesc);
template __global__ void axis_pass_pipe<float,512,false,8,900,60,15,10,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,512,true,0,900,60,15,10,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,1125,75,15,15,5>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,1125,75,15,15,5>(const PassDesc);
template __global__ void axis_pass_static<float,true,1024,1296,216,6,6,6,6>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,1296,216,6,6,6,6>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,1600,100,10,10,16>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,1600,100,10,10,16>(const PassDesc);
template __global__ void axis_pass_static<float,true,1024,1944,324,6,6,6,3,3>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,1944,324,6,6,6,3,3>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,2250,150,15,15,10>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,2250,150,15,15,10>(const PassDesc);
template __global__ void axis_pass_static<float,true,1024,2592,216,12,6,6,6>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,2592,216,12,6,6,6>(const PassDesc);
template __global__ void axis_pass_static<float,true,1024,3125,625,5,5,5,5,5>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,3125,625,5,5,5,5,5>(const PassDesc);
template __global__ void axis_pass_static<float,true,1024,3645,243,15,3,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,3645,243,15,3,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<float,true,1024,4096,256,16,16,16>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,4096,256,16,16,16>(const PassDesc);
extern const StaticPlan kPlans_f32_4[];
extern const int kPlansCount_f32_4;
const StaticPlan kPlans_f32_4[] = {
  {5, 1, 1, {5}, 1024, (const void*)&axis_pass_static<float,true,1024,5,1,5>, (const void*)&axis_pass_static<float,false,1024,5,1,5>, nullptr, nullptr, 1024, 0},
  {15, 1, 1, {15}, 1024, (const void*)&axis_pass_static<float,true,1024,15,1,15>, (const void*)&axis_pass_static<float,false,1024,15,1,15>, (const void*)&axis_pass_pipe<float,1024,false,16,15,1,15>, (const void*)&axis_pass_pipe<float,1024,true,0,15,1,15>, 1024, 16},
  {27, 9, 3, {3,3,3}, 1024, (const void*)&axis_pass_static<float,true,1024,27,9,3,3,3>, (const void*)&axis_pass_static<float,false,1024,27,9,3,3,3>, (const void*)&axis_pass_pipe<float,1024,false,16,27,9,3,3,3>, (const void*)&axis_pass_pipe<float,1024,true,0,27,9,3,3,3>, 1024, 16},
  {48, 6, 2, {6,8}, 1024, (const void*)&axis_pass_static<float,true,1024,48,6,6,8>, (const void*)&axis_pass_static<float,false,1024,48,6,6,8>, (const void*)&axis_pass_pipe<float,1024,false,16,48,6,6,8>, (const void*)&axis_pass_pipe<float,1024,true,0,48,6,6,8>, 1024, 16},
  {75, 5, 2, {15,5}, 1024, (const void*)&axis_pass_static<float,true,1024,75,5,15,5>, (const void*)&axis_pass_static<float,false,1024,75,5,15,5>, (const void*)&axis_pass_pipe<float,1024,false,16,75,5,15,5>, (const void*)&axis_pass_pipe<float,1024,true,0,75,5,15,5>, 1024, 16},
  {108, 18, 3, {6,6,3}, 1024, (const void*)&axis_pass_static<float,true,1024,108,18,6,6,3>, (const void*)&axis_pass_static<float,false,1024,108,18,6,6,3>, (const void*)&axis_pass_pipe<float,1024,false,16,108,18,6,6,3>, (const void*)&axis_pass_pipe<float,1024,true,0,108,18,6,6,3>, 1024, 16},
  {150, 10, 2, {15,10}, 512, (const void*)&axis_pass_static<float,true,512,150,10,15,10>, (const void*)&axis_pass_static<float,false,512,150,10,15,10>, (const void*)&axis_pass_pipe<float,512,false,16,150,10,15,10>, (const void*)&axis_pass_pipe<float,512,true,0,150,10,15,10>, 512, 16},
  {216, 36, 3, {6,6,6}, 1024, (const void*)&axis_pass_static<float,true,1024,216,36,6,6,6>, (const void*)&axis_pass_static<float,false,1024,216,36,6,6,6>, (const void*)&axis_pass_pipe<float,1024,false,16,216,36,6,6,6>, (const void*)&axis_pass_pipe<float,1024,true,0,216,36,6,6,6>, 1024, 16},
  {270, 18, 3, {15,6,3}, 512, (const void*)&axis_pass_static<float,true,512,270,18,15,6,3>, (const void*)&axis_pass_static<float,false,512,270,18,15,6,3>, (const void*)&axis_pass_pipe<float,512,false,16,270,18,15,6,3>, (const void*)&axis_pass_pipe<float,512,true,0,270,18,15,6,3>, 512, 16},
  {375, 25, 3, {15,5,5}, 1024, (const void*)&axis_pass_static<float,true,1024,375,25,15,5,5>, (const void*)&axis_pass_static<float,false,1024,375,25,15,5,5>, (const void*)&axis_pass_pipe<float,1024,false,16,375,25,15,5,5>, (const void*)&axis_pass_pipe<float,1024,true,0,375,25,15,5,5>, 1024, 16},
  {480, 48, 3, {10,6,8}, 1024, (const void*)&axis_pass_static<float,true,1024,480,48,10,6,8>, (const void*)&axis_pass_static<float,false,1024,480,48,10,6,8>, (const void*)&axis_pass_pipe<float,1024,false,16,480,48,10,6,8>, (const void*)&axis_pass_pipe<float,1024,true,0,480,48,10,6,8>, 1024, 16},
  {600, 60, 3, {10,10,6}, 1024, (const void*)&axis_pass_static<float,true,1024,600,60,10,10,6>, (const void*)&axis_pass_static<float,false,1024,600,60,10,10,6>, (const void*)&axis_pass_pipe<float,1024,false,16,600,60,10,10,6>, (const void*)&axis_pass_pipe<float,1024,true,0,600,60,10,10,6>, 1024, 16},
  {729, 243, 6, {3,3,3,3,3,3}, 1024, (const void*)&axis_pass_static<float,true,1024,729,243,3,3,3,3,3,3>, (const void*)&axis_pass_static<float,false,1024,729,243,3,3,3,3,3,3>, (const void*)&axis_pass_pipe<float,1024,false,4,729,243,3,3,3,3,3,3>, (const void*)&axis_pass_pipe<float,1024,true,0,729,243,3,3,3,3,3,3>, 1024, 4},
  {900, 60, 3, {15,10,6}, 512, (const void*)&axis_pass_static<float,true,512,900,60,15,10,6>, (const void*)&axis_pass_static<float,false,512,900,60,15,10,6>, (const void*)&axis_pass_pipe<float,512,false,8,900,60,15,10,6>, (const void*)&axis_pass_pipe<float,512,true,0,900,60,15,10,6>, 512, 8},
  {1125, 75, 3, {15,15,5}, 1024, (const void*)&axis_pass_static<float,true,1024,1125,75,15,15,5>, (const void*)&axis_pass_static<float,false,1024,1125,75,15,15,5>, nullptr, nullptr, 1024, 0},
  {1296, 216, 4, {6,6,6,6}, 1024, (const void*)&axis_pass_static<float,true,1024,1296,216,6,6,6,6>, (const void*)&axis_pass_static<float,false,1024,1296,216,6,6,6,6>, nullptr, nullptr, 1024, 0},
  {1600, 100, 3, {10,10,16}, 512, (const void*)&axis_pass_static<float,true,512,1600,100,10,10,16>, (const void*)&axis_pass_static<float,false,512,1600,100,10,10,16>, nullptr, nullptr, 512, 0},
  {1944, 324, 5, {6,6,6,3,3}, 1024, (const void*)&axis_pass_static<float,true,1024,1944,324,6,6,6,3,3>, (const void*)&axis_pass_static<float,false,1024,1944,324,6,6,6,3,3>, nullptr, nullptr, 1024, 0},
  {2250, 150, 3, {15,15,10}, 512, (const void*)&axis_pass_static<float,true,512,2250,150,15,15,10>, (const void*)&axis_pass_static<float,false,512,2250,150,15,15,10>, nullptr, nullptr, 512, 0},
  {2592, 216, 4, {12,6,6,6}, 1024, (const void*)&axis_pass_static<float,true,1024,2592,216,12,6,6,6>, (const void*)&axis_pass_static<float,false,1024,2592,216,12,6,6,6>, nullptr, nullptr, 1024, 0},
  {3125, 625, 5, {5,5,5,5,5}, 1024, (const void*)&axis_pass_static<float,true,1024,3125,625,5,5,5,5,5>, (const void*)&axis_pass_static<float,false,1024,3125,625,5,5,5,5,5>, nullptr, nullptr, 1024, 0},
  {3645, 243, 6, {15,3,3,3,3,3}, 1024, (const void*)&axis_pass_static<float,true,1024,3645,243,15,3,3,3,3,3>, (const void*)&axis_pass_static<float,false,1024,3645,243,15,3,3,3,3,3>, nullptr, nullptr, 1024, 0},
  {4096, 256, 3, {16,16,16}, 1024, (const void*)&axis_pass_static<float,true,1024,4096,256,16,16,16>, (const void*)&axis_pass_static<float,false,1024,4096,256,16,16,16>, nullptr, nullptr, 1024, 0},
};
const int kPlansCount_f32_4 = 23;
}  // namespace dfft
