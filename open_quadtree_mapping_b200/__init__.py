"""B200-native per-keyframe depth pipeline of QuadtreeMapping (quadmap::Depthmap)."""
