// Generated by gen_plans.py -- do not edit.
#include "static_plans.h"
namespace dfft {
template __global__ void axis_pass_static<double,true,1024,1,1,1>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,1,1,1>(const PassDesc);
template __global__ void axis_pass_static<double,true,1024,8,1,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,8,1,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,8,1,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,8,1,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,18,3,6,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,18,3,6,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,18,3,6,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,18,3,6,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,32,4,8,4>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,32,4,8,4>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,32,4,8,4>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,32,4,8,4>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,54,9,6,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,54,9,6,3,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,54,9,6,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,54,9,6,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,81,27,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,81,27,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,81,27,3,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,81,27,3,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,125,25,5,5,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,125,25,5,5,5>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,125,25,5,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,125,25,5,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,162,27,6,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,162,27,6,3,3,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,162,27,6,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,162,27,6,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,256,240,15,15,16>(const PassDesc);
template __global__ void axis_pass_static<double,false,256,240,15,15,16>(const PassDesc);
template __global__ void axis_pass_pipe<double,256,false,8,240,15,15,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,256,true,0,240,15,15,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,300,30,10,6,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,300,30,10,6,5>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,300,30,10,6,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,300,30,10,6,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,400,40,10,5,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,400,40,10,5,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,400,40,10,5,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,400,40,10,5,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,500,50,10,10,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,500,50,10,10,5>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,500,50,10,10,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,500,50,10,10,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,640,64,10,8,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,640,64,10,8,8>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,768,64,12,8,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,768,64,12,8,8>(const PassDesc);
template __global__ void axis_pass_static<double,true,1024,972,162,6,6,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,972,162,6,6,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1200,100,12,10,10>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1200,100,12,10,10>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1440,120,12,12,10>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1440,120,12,12,10>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1728,144,12,12,12>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1728,144,12,12,12>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,2025,135,15,15,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,2025,135,15,15,3,3>(const PassDesc);
extern const StaticPlan kPlans_f64_0[];
extern const int kPlansCount_f64_0;
const StaticPlan kPlans_f64_0[] = {
  {1, 1, 1, {1}, 1024, (const void*)&axis_pass_static<double,true,1024,1,1,1>, (const void*)&axis_pass_static<double,false,1024,1,1,1>, nullptr, nullptr, 512, 0},
  {8, 1, 1, {8}, 1024, (const void*)&axis_pass_static<double,true,1024,8,1,8>, (const void*)&axis_pass_static<double,false,1024,8,1,8>, (const void*)&axis_pass_pipe<double,512,false,8,8,1,8>, (const void*)&axis_pass_pipe<double,512,true,0,8,1,8>, 512, 8},
  {18, 3, 2, {6,3}, 1024, (const void*)&axis_pass_static<double,true,1024,18,3,6,3>, (const void*)&axis_pass_static<double,false,1024,18,3,6,3>, (const void*)&axis_pass_pipe<double,512,false,8,18,3,6,3>, (const void*)&axis_pass_pipe<double,512,true,0,18,3,6,3>, 512, 8},
  {32, 4, 2, {8,4}, 1024, (const void*)&axis_pass_static<double,true,1024,32,4,8,4>, (const void*)&axis_pass_static<double,false,1024,32,4,8,4>, (const void*)&axis_pass_pipe<double,512,false,8,32,4,8,4>, (const void*)&axis_pass_pipe<double,512,true,0,32,4,8,4>, 512, 8},
  {54, 9, 3, {6,3,3}, 1024, (const void*)&axis_pass_static<double,true,1024,54,9,6,3,3>, (const void*)&axis_pass_static<double,false,1024,54,9,6,3,3>, (const void*)&axis_pass_pipe<double,512,false,8,54,9,6,3,3>, (const void*)&axis_pass_pipe<double,512,true,0,54,9,6,3,3>, 512, 8},
  {81, 27, 4, {3,3,3,3}, 1024, (const void*)&axis_pass_static<double,true,1024,81,27,3,3,3,3>, (const void*)&axis_pass_static<double,false,1024,81,27,3,3,3,3>, (const void*)&axis_pass_pipe<double,512,false,8,81,27,3,3,3,3>, (const void*)&axis_pass_pipe<double,512,true,0,81,27,3,3,3,3>, 512, 8},
  {125, 25, 3, {5,5,5}, 1024, (const void*)&axis_pass_static<double,true,1024,125,25,5,5,5>, (const void*)&axis_pass_static<double,false,1024,125,25,5,5,5>, (const void*)&axis_pass_pipe<double,512,false,8,125,25,5,5,5>, (const void*)&axis_pass_pipe<double,512,true,0,125,25,5,5,5>, 512, 8},
  {162, 27, 4, {6,3,3,3}, 1024, (const void*)&axis_pass_static<double,true,1024,162,27,6,3,3,3>, (const void*)&axis_pass_static<double,false,1024,162,27,6,3,3,3>, (const void*)&axis_pass_pipe<double,512,false,8,162,27,6,3,3,3>, (const void*)&axis_pass_pipe<double,512,true,0,162,27,6,3,3,3>, 512, 8},
  {240, 15, 2, {15,16}, 256, (const void*)&axis_pass_static<double,true,256,240,15,15,16>, (const void*)&axis_pass_static<double,false,256,240,15,15,16>, (const void*)&axis_pass_pipe<double,256,false,8,240,15,15,16>, (const void*)&axis_pass_pipe<double,256,true,0,240,15,15,16>, 256, 8},
  {300, 30, 3, {10,6,5}, 512, (const void*)&axis_pass_static<double,true,512,300,30,10,6,5>, (const void*)&axis_pass_static<double,false,512,300,30,10,6,5>, (const void*)&axis_pass_pipe<double,512,false,8,300,30,10,6,5>, (const void*)&axis_pass_pipe<double,512,true,0,300,30,10,6,5>, 512, 8},
  {400, 40, 3, {10,5,8}, 512, (const void*)&axis_pass_static<double,true,512,400,40,10,5,8>, (const void*)&axis_pass_static<double,false,512,400,40,10,5,8>, (const void*)&axis_pass_pipe<double,512,false,8,400,40,10,5,8>, (const void*)&axis_pass_pipe<double,512,true,0,400,40,10,5,8>, 512, 8},
  {500, 50, 3, {10,10,5}, 512, (const void*)&axis_pass_static<double,true,512,500,50,10,10,5>, (const void*)&axis_pass_static<double,false,512,500,50,10,10,5>, (const void*)&axis_pass_pipe<double,512,false,8,500,50,10,10,5>, (const void*)&axis_pass_pipe<double,512,true,0,500,50,10,10,5>, 512, 8},
  {640, 64, 3, {10,8,8}, 512, (const void*)&axis_pass_static<double,true,512,640,64,10,8,8>, (const void*)&axis_pass_static<double,false,512,640,64,10,8,8>, nullptr, nullptr, 512, 0},
  {768, 64, 3, {12,8,8}, 512, (const void*)&axis_pass_static<double,true,512,768,64,12,8,8>, (const void*)&axis_pass_static<double,false,512,768,64,12,8,8>, nullptr, nullptr, 512, 0},
  {972, 162, 5, {6,6,3,3,3}, 1024, (const void*)&axis_pass_static<double,true,1024,972,162,6,6,3,3,3>, (const void*)&axis_pass_static<double,false,1024,972,162,6,6,3,3,3>, nullptr, nullptr, 512, 0},
  {1200, 100, 3, {12,10,10}, 512, (const void*)&axis_pass_static<double,true,512,1200,100,12,10,10>, (const void*)&axis_pass_static<double,false,512,1200,100,12,10,10>, nullptr, nullptr, 512, 0},
  {1440, 120, 3, {12,12,10}, 512, (const void*)&axis_pass_static<double,true,512,1440,120,12,12,10>, (const void*)&axis_pass_static<double,false,512,1440,120,12,12,10>, nullptr, nullptr, 512, 0},
  {1728, 144, 3, {12,12,12}, 512, (const void*)&axis_pass_static<double,true,512,1728,144,12,12,12>, (const void*)&axis_pass_static<double,false,512,1728,144,12,12,12>, nullptr, nullptr, 512, 0},
  {2025, 135, 4, {15,15,3,3}, 512, (const void*)&axis_pass_static<double,true,512,2025,135,15,15,3,3>, (const void*)&axis_pass_static<double,false,512,2025,135,15,15,3,3>, nullptr, nullptr, 512, 0},
};
const int kPlansCount_f64_0 = 19;
}  // namespace dfft
