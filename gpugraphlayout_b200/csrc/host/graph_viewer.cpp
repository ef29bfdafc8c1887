// graph_viewer.cpp -- the command line of the reference (src/graph_viewer.cpp)
// on the B200 engine:
//
//   graph_viewer gpu|cpu max_iterations num_snaps sg|wg scale gravity
//                exact|approximate edgelist_path out_path [png w h|csv|bin]
//
// Same arguments, checks, output names (<edgelist basename>_<iter>.<fmt>) and
// progress lines.  Differences: this build provides the GPU path only, so
// `cpu` is refused with a message; with exactly ten arguments the format
// defaults to png (the reference reads argv[10] past the end there).  png
// output is rendered on the GPU and written by this library's PNG encoder.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <string>

#include "RPCommon.hpp"
#include "RPGPUForceAtlas2.hpp"
#include "RPGraph.hpp"
#include "RPGraphLayout.hpp"

int main(int argc, const char **argv)
{
    srandom(1234);  // src/graph_viewer.cpp:49

    if (argc < 10 || (argc > 10 && std::string(argv[10]) == "png" && argc < 13)) {
        fprintf(stderr, "Usage: graph_viewer gpu|cpu max_iterations num_snaps sg|wg scale gravity "
                        "exact|approximate edgelist_path out_path [png image_w image_h|csv|bin]\n");
        exit(EXIT_FAILURE);
    }

    const bool cuda_requested = std::string(argv[1]) == "gpu" || std::string(argv[1]) == "cuda";
    const int max_iterations = std::stoi(argv[2]);
    const int num_screenshots = std::stoi(argv[3]);
    const bool strong_gravity = std::string(argv[4]) == "sg";
    const float scale = std::stof(argv[5]);
    const float gravity = std::stof(argv[6]);
    const bool approximate = std::string(argv[7]) == "approximate";
    std::string edgelist_path = argv[8];
    std::string out_path = argv[9];
    std::string out_format = "png";
    int image_w = 1250, image_h = 1250;

    for (int arg_no = 10; arg_no < argc; arg_no++) {
        const std::string a = argv[arg_no];
        if (a == "png") {
            out_format = "png";
            image_w = std::stoi(argv[arg_no + 1]);
            image_h = std::stoi(argv[arg_no + 2]);
            arg_no += 2;
        } else if (a == "csv") {
            out_format = "csv";
        } else if (a == "bin") {
            out_format = "bin";
        }
    }

    if (cuda_requested && !approximate) {
        fprintf(stderr, "error: The CUDA implementation (currently) requires Barnes-Hut approximation.\n");
        exit(EXIT_FAILURE);
    }
    if (!is_file_exists(edgelist_path)) {
        fprintf(stderr, "error: No edgelist at %s\n", edgelist_path.c_str());
        exit(EXIT_FAILURE);
    }
    if (!is_file_exists(out_path)) {
        fprintf(stderr, "error: No output folder at %s\n", out_path.c_str());
        exit(EXIT_FAILURE);
    }
    if (!cuda_requested) {
        fprintf(stderr, "error: this build provides the GPU (gpu|cuda) path only.\n");
        exit(EXIT_FAILURE);
    }

    printf("Loading edgelist at '%s'...", edgelist_path.c_str());
    fflush(stdout);
    RPGraph::UGraph graph(edgelist_path);
    printf("done.\n");
    printf("    fetched %d nodes and %d edges.\n", graph.num_nodes(), graph.num_edges());

    RPGraph::GraphLayout layout(graph);
    RPGraph::ForceAtlas2 *fa2 =
        new RPGraph::CUDAForceAtlas2(layout, approximate, strong_gravity, gravity, scale);

    printf("Started Layout algorithm...\n");
    const int snap_period = ceil((float)max_iterations / num_screenshots);
    const int print_period = ceil((float)max_iterations * 0.05);

    for (int iteration = 1; iteration <= max_iterations; ++iteration) {
        fa2->doStep();
        if (num_screenshots > 0 && (iteration % snap_period == 0 || iteration == max_iterations)) {
            std::string edgelist_basename = basename(edgelist_path);
            std::string out_filename =
                edgelist_basename + "_" + std::to_string(iteration) + "." + out_format;
            std::string out_filepath = out_path + "/" + out_filename;
            printf("Starting iteration %d (%.2f%%), writing %s...", iteration,
                   100 * (float)iteration / max_iterations, out_format.c_str());
            fflush(stdout);
            fa2->sync_layout();
            if (out_format == "png")
                layout.writeToPNG(image_w, image_h, out_filepath);
            else if (out_format == "csv")
                layout.writeToCSV(out_filepath);
            else if (out_format == "bin")
                layout.writeToBin(out_filepath);
            printf("done.\n");
        } else if (print_period > 0 && iteration % print_period == 0) {
            printf("Starting iteration %d (%.2f%%).\n", iteration,
                   100 * (float)iteration / max_iterations);
        }
    }

    delete fa2;
    exit(EXIT_SUCCESS);
}
